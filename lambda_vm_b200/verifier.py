"""STARK verifier for the multi-table proofs of lambda_vm_b200.stark.

Restates the checks of crypto/stark/src/verifier.rs (multi_verify): per-table
transcript replay, the bus balance of the LogUp contributions, the step-2
composition check at the out-of-domain point (H(z) = H0(z^2) + z H1(z^2)
against the constraints evaluated on the OOD frame), the step-3 FRI checks
(layer openings and authentication paths, fold consistency, the terminal
polynomial) and the grinding nonce, with the library's Keccak-256 and
transcript and Python-integer field arithmetic on the host. Returns
(ok, reason). `verify_bytes` takes a serialized proof (proof_io).
"""
import numpy as np

from . import field as F
from . import math_cuda as mc

P = F.P
GRIND_PREFIX = bytes([0x01, 0x23, 0x45, 0x67, 0x89, 0xAB, 0xCD, 0xED])  # grinding.rs:6


def f3(x):
    return tuple(int(v) % P for v in x)


def add(a, b):
    return tuple((a[i] + b[i]) % P for i in range(3))


def sub(a, b):
    return tuple((a[i] - b[i]) % P for i in range(3))


def mul(a, b):
    a0, a1, a2 = a
    b0, b1, b2 = b
    return ((a0 * b0 + 2 * (a1 * b2 + a2 * b1)) % P, (a0 * b1 + a1 * b0 + 2 * a2 * b2) % P,
            (a0 * b2 + a1 * b1 + a2 * b0) % P)


def scale(a, s):
    return tuple(v * (s % P) % P for v in a)


def fpow(a, e):
    r, b = (1, 0, 0), f3(a)
    while e:
        if e & 1:
            r = mul(r, b)
        b = mul(b, b)
        e >>= 1
    return r


def finv(a):
    a0, a1, a2 = f3(a)
    nrm = (a0 ** 3 + 2 * a1 ** 3 + 4 * a2 ** 3 - 6 * a0 * a1 * a2) % P
    ni = pow(nrm, P - 2, P)
    return ((a0 * a0 - 2 * a1 * a2) * ni % P, (2 * a2 * a2 - a0 * a1) * ni % P, (a1 * a1 - a0 * a2) * ni % P)


def brev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


def root(log_n):
    return F.root_of_unity(log_n) % P


def merkle_ok(leaf_hash, idx, path, rt):
    h = leaf_hash
    for sib in path:
        s = bytes(sib)
        h = mc.keccak256(h + s) if idx % 2 == 0 else mc.keccak256(s + h)
        idx //= 2
    return h == rt


def row_pair_leaf(r0, r1):
    b = b""
    for row in (r0, r1):
        for v in row:
            b += (int(v) % P).to_bytes(8, "big")
    return mc.keccak256(b)


def eval_ood(prog, frame, rap, alpha, offset):
    """Constraint roots at the OOD point; frame[off][col] over main || aux."""
    v = []
    m_main = frame["m"]
    for nd in prog["nodes"]:
        k = nd[0]
        if k == "var":
            _, is_main, off, col = nd
            v.append(frame["vals"][off][col if is_main else m_main + col])
        elif k == "cb":
            v.append((prog["base_consts"][nd[1]] % P, 0, 0))
        elif k == "ce":
            v.append(f3(prog["ext_consts"][nd[1]]))
        elif k == "rap":
            v.append(f3(rap[nd[1]]))
        elif k == "alpha":
            v.append(f3(alpha[nd[1]]))
        elif k == "off":
            v.append(f3(offset))
        elif k == "add":
            v.append(add(v[nd[1]], v[nd[2]]))
        elif k == "sub":
            v.append(sub(v[nd[1]], v[nd[2]]))
        elif k == "mul":
            v.append(mul(v[nd[1]], v[nd[2]]))
        elif k == "neg":
            v.append(scale(v[nd[1]], P - 1))
        else:
            v.append(v[nd[1]])
    return [v[r] for r in prog["roots"]]


def public_sum(terms, z, apows):
    """The verifier's side of LogUp buses with public content (a program's
    instructions and execution counts, a claimed output): sum of m / (z -
    (bus + sum_i alpha^(i+1) v_i)) over (bus, values, signed m) terms."""
    s = (0, 0, 0)
    for bus, vals, m in terms:
        fp = sub(z, (bus % P, 0, 0))
        for i, v in enumerate(vals):
            fp = sub(fp, scale(apows[i + 1], int(v)))
        s = add(s, scale(finv(fp), m % P))
    return s


def verify(airs, proof, opts, label=b"lambda_vm_b200/synthetic-multi-table", device=None, public_terms=()):
    """Verify a multi-table proof: (ok, reason). With `device` (a context from
    device.backend()) the query phase runs on the GPU (sg_verify_queries).
    `public_terms` are bus terms whose content the statement fixes
    (public_sum); they join the tables' contributions in the bus balance. A
    proof of the wrong shape (missing fields, short vectors) is rejected."""
    try:
        ok, reason, prep = _replay(airs, proof, opts, label, public_terms)
        if not ok:
            return ok, reason
        if device is not None:
            return verify_queries_gpu([prep], device)[0]
        for pr in prep:
            ok, reason = _check_queries_host(pr)
            if not ok:
                return ok, reason
    except (IndexError, KeyError, TypeError, ValueError) as e:
        return False, f"malformed proof: {type(e).__name__}"
    return True, "ok"


def _replay(airs, proof, opts, label, public_terms=()):
    """Transcript replay and every check that needs it (bus balance, the
    composition identity at z, FRI layer count, terminal length, grinding,
    query indexes); returns (ok, reason, per-table values for the query phase)."""
    T = mc.Transcript(label)
    tabs = proof["tables"]
    if len(tabs) != len(airs):
        # every table of the proof is checked against an AIR of the statement
        return False, "the proof's table count is not the statement's", None
    for tp in tabs:
        T.append_bytes(tp["main_root"])
    ch = [f3(T.sample_ext3()), f3(T.sample_ext3())]
    alpha = ch[1]
    apows = [(1, 0, 0)]
    for _ in range(max(a.max_alpha for a in airs) - 1):
        apows.append(mul(apows[-1], alpha))
    total = public_sum(public_terms, ch[0], apows)
    for tp in tabs:
        total = add(total, f3(tp["table_contribution"]))
    if total != (0, 0, 0):
        return False, "bus contributions do not balance", None
    prep = []
    B, g = opts.blowup, opts.coset_offset
    for ti, (air, tp) in enumerate(zip(airs, tabs)):
        t = T.clone()
        if len(tabs) > 1:
            t.append_bytes(int(ti).to_bytes(8, "little"))
        n = air.n
        N = n * B
        logN = N.bit_length() - 1
        t.append_bytes(tp["aux_root"])
        beta = f3(t.sample_ext3())
        prog = air.program
        ncons = len(prog["roots"]) + len(air.boundary)
        coefs = [(1, 0, 0)]
        for _ in range(ncons - 1):
            coefs.append(mul(coefs[-1], beta))
        bt, bb = coefs[:len(prog["roots"])], coefs[len(prog["roots"]):]
        t.append_bytes(tp["comp_root"])
        z = f3(t.sample_z_ood(n, N, g))
        wn = root(air.log_n)
        zw = scale(z, wn)
        z2 = mul(z, z)
        tood = [[f3(v) for v in tp["trace_ood"][k]] for k in range(2)]
        pood = [f3(v) for v in tp["parts_ood"]]
        # step 2: composition identity at z
        L = f3(tp["table_contribution"])
        offset = scale(L, pow(n, P - 2, P))
        frame = {"m": air.width, "vals": tood}
        roots_v = eval_ood(prog, frame, ch, apows, offset)
        acc = (0, 0, 0)
        for c, cv in enumerate(roots_v):
            acc = add(acc, mul(bt[c], cv))
        zn1 = sub(fpow(z, n), (1, 0, 0))
        h = mul(acc, finv(zn1))
        for b, (col, is_aux, row) in enumerate(air.boundary):
            cell = tood[0][air.width + col] if is_aux else tood[0][col]
            h = add(h, mul(mul(bb[b], cell), finv(sub(z, (1, 0, 0)))))
        if h != add(pood[0], mul(z, pood[1])):
            return False, f"table {ti}: composition check failed", None
        for k in range(2):
            for v in tood[k]:
                t.append_ext3(np.array(v, np.uint64))
        for v in pood:
            t.append_ext3(np.array(v, np.uint64))
        gamma = f3(t.sample_ext3())
        ncols = air.width + air.aux_width
        gp = [(1, 0, 0)]
        for _ in range(2 + 2 * ncols - 1):
            gp.append(mul(gp[-1], gamma))
        gh, gt = gp[:2], gp[2:]
        # FRI transcript replay
        blog = B.bit_length() - 1
        terminal_log = min(blog + opts.final_log_degree, logN)
        total_folds = logN - terminal_log
        num_committed = max(total_folds - 1, 0)
        if len(tp["fri_roots"]) != num_committed:
            return False, "wrong number of FRI layers", None
        zetas = []
        for li in range(num_committed):
            zetas.append(f3(t.sample_ext3()))
            t.append_bytes(tp["fri_roots"][li])
        if total_folds > 0:
            zetas.append(f3(t.sample_ext3()))
        coeffs = [f3(c) for c in tp["fri_final_coeffs"]]
        if len(coeffs) != 1 << (terminal_log - blog):
            return False, "wrong terminal length", None
        for c in coeffs:
            t.append_ext3(np.array(c, np.uint64))
        if opts.grinding:
            inner = mc.keccak256(GRIND_PREFIX + t.state() + bytes([opts.grinding]))
            head = int.from_bytes(mc.keccak256(inner + int(tp["nonce"]).to_bytes(8, "big"))[:8], "big")
            if head >= 1 << (64 - opts.grinding):
                return False, "grinding nonce invalid", None
            t.append_bytes(int(tp["nonce"]).to_bytes(8, "big"))
        iotas = [t.sample_u64(N // 2) for _ in range(opts.queries)]
        if list(iotas) != list(tp["iotas"]):
            return False, "query indexes differ", None
        prep.append({"air": air, "tp": tp, "g": g, "n": n, "N": N, "logN": logN, "z": z, "zw": zw, "z2": z2,
                     "tood": tood, "pood": pood, "gh": gh, "gt": gt, "zetas": zetas, "coeffs": coeffs,
                     "total_folds": total_folds, "num_committed": num_committed, "terminal_log": terminal_log,
                     "iotas": iotas, "ncols": ncols})
    return True, "ok", prep


def _check_queries_host(pr):
    """The query phase of one table on the host (Python integers)."""
    air, tp, g, logN = pr["air"], pr["tp"], pr["g"], pr["logN"]
    z, zw, z2, tood, pood, gh, gt = pr["z"], pr["zw"], pr["z2"], pr["tood"], pr["pood"], pr["gh"], pr["gt"]
    zetas, coeffs, ncols = pr["zetas"], pr["coeffs"], pr["ncols"]
    total_folds, num_committed, terminal_log = pr["total_folds"], pr["num_committed"], pr["terminal_log"]
    wN = root(logN)
    term_off = pow(g, 1 << total_folds, P)
    wT = root(terminal_log)
    for q, iota in enumerate(pr["iotas"]):
        r0, r1 = brev(2 * iota, logN), brev(2 * iota + 1, logN)
        om, oa, op = tp["open_main"], tp["open_aux"], tp["open_parts"]
        if not merkle_ok(row_pair_leaf(om[2 * q], om[2 * q + 1]), iota, tp["path_main"][q], tp["main_root"]):
            return False, "main opening path"
        if not merkle_ok(row_pair_leaf(oa[2 * q], oa[2 * q + 1]), iota, tp["path_aux"][q], tp["aux_root"]):
            return False, "aux opening path"
        if not merkle_ok(row_pair_leaf(op[2 * q], op[2 * q + 1]), iota, tp["path_parts"][q], tp["comp_root"]):
            return False, "parts opening path"
        dv = []
        for rr, r in ((2 * q, r0), (2 * q + 1, r1)):
            x = g * pow(wN, r, P) % P
            ih = finv(sub((x, 0, 0), z2))
            acc = (0, 0, 0)
            for j in range(2):
                hx = f3(op[rr][3 * j:3 * j + 3])
                acc = add(acc, mul(mul(gh[j], sub(hx, pood[j])), ih))
            for kk, pt in enumerate((z, zw)):
                it = finv(sub((x, 0, 0), pt))
                for j in range(ncols):
                    tv = (int(om[rr][j]) % P, 0, 0) if j < air.width else f3(oa[rr][3 * (j - air.width):3 * (j - air.width) + 3])
                    acc = add(acc, mul(mul(gt[2 * j + kk], sub(tv, tood[kk][j])), it))
            dv.append(acc)
        # fold chain
        x0 = g * pow(wN, brev(iota, logN - 1), P) % P
        if x0 != g * pow(wN, r0, P) % P:
            return False, "query point mismatch"
        v = add(add(dv[0], dv[1]), scale(mul(zetas[0], sub(dv[0], dv[1])), pow(x0, P - 2, P))) if total_folds else None
        for li in range(num_committed):
            f = li + 1
            pos = iota >> li
            leaf = pos >> 1
            pair = tp["fri_open"][li][2 * q:2 * q + 2]
            a, b = f3(pair[0]), f3(pair[1])
            if (a, b)[pos & 1] != v:
                return False, f"FRI layer {f} value mismatch"
            lb = b"".join((int(u) % P).to_bytes(8, "big") for u in list(pair[0]) + list(pair[1]))
            if not merkle_ok(mc.keccak256(lb), leaf, tp["fri_paths"][li][q], tp["fri_roots"][li]):
                return False, f"FRI layer {f} path"
            xj = pow(g * pow(wN, brev(leaf << f, logN - 1), P) % P, 1 << f, P)
            v = add(add(a, b), scale(mul(zetas[f], sub(a, b)), pow(xj, P - 2, P)))
        if total_folds:
            p_term = iota >> (total_folds - 1)
            xt = term_off * pow(wT, brev(p_term, terminal_log), P) % P
            ev = (0, 0, 0)
            for c in reversed(coeffs):
                ev = add(scale(ev, xt), c)
            if ev != v:
                return False, "terminal polynomial mismatch"
    return True, "ok"


_REASONS = {1: "main opening path", 2: "aux opening path", 3: "parts opening path",
            4: "FRI layer {} value mismatch", 5: "FRI layer {} path", 6: "terminal polynomial mismatch"}


def verify_queries_gpu(preps, be):
    """The query phase of every table of every proof in `preps` (a list of
    _replay results) in one sg_verify_queries launch; one (ok, reason) per
    proof, the reason of its first failing query as the host check gives it."""
    import ctypes as C
    from . import native
    from .device import DeviceBuffer
    blob = bytearray()

    def put(arr):
        b = bytes(arr)
        off = len(blob)
        blob.extend(b)
        blob.extend(b"\0" * (-len(blob) % 8))
        return off

    def u64(vals):
        return np.ascontiguousarray(np.asarray(vals, dtype=np.uint64).reshape(-1)).tobytes()

    def u8(vals):
        return np.ascontiguousarray(np.asarray(vals, dtype=np.uint8).reshape(-1)).tobytes()

    flat, owners, offs = [], [], []
    for pi, prep in enumerate(preps):
        for pr in prep:
            tp = pr["tp"]
            W = pr["ncols"]
            consts = [pr["z"], pr["zw"], pr["z2"]] + list(pr["gh"]) + list(pr["pood"]) + list(pr["gt"])
            consts += list(pr["tood"][0]) + list(pr["tood"][1]) + list(pr["zetas"]) + list(pr["coeffs"])
            assert len(consts) == 7 + 4 * W + pr["total_folds"] + len(pr["coeffs"])
            o = {"consts": put(u64(consts)),
                 "roots": put(b"".join(bytes(r) for r in [tp["main_root"], tp["aux_root"], tp["comp_root"]] +
                                       list(tp["fri_roots"]))),
                 "iotas": put(u64(pr["iotas"])), "open_main": put(u64(tp["open_main"])),
                 "open_aux": put(u64(tp["open_aux"])), "open_parts": put(u64(tp["open_parts"])),
                 "path_main": put(u8(tp["path_main"])), "path_aux": put(u8(tp["path_aux"])),
                 "path_parts": put(u8(tp["path_parts"])),
                 "fri_open": put(b"".join(u64(x) for x in tp["fri_open"])),
                 "fri_paths": put(b"".join(u8(x) for x in tp["fri_paths"]))}
            flat.append(pr)
            owners.append(pi)
            offs.append(o)
    out = [(True, "ok")] * len(preps)
    if not flat:
        return out
    dev = DeviceBuffer.from_host(np.frombuffer(bytes(blob), np.uint8), be)
    try:
        tabs = (native.VerifyTable * len(flat))()
        for i, (pr, o) in enumerate(zip(flat, offs)):
            air = pr["air"]
            t = tabs[i]
            t.log_n, t.log_N, t.m, t.aux_cols = air.log_n, pr["logN"], air.width, air.aux_width
            t.queries, t.fri_layers = len(pr["iotas"]), pr["num_committed"]
            t.total_folds, t.terminal_log, t.num_coeffs = pr["total_folds"], pr["terminal_log"], len(pr["coeffs"])
            t.coset_offset, t.omega_N = pr["g"], root(pr["logN"])
            t.terminal_offset, t.omega_T = pow(pr["g"], 1 << pr["total_folds"], P), root(pr["terminal_log"])
            for name, off in o.items():
                setattr(t, name, dev.ptr + off)
        total = sum(len(pr["iotas"]) for pr in flat)
        status = np.zeros(max(total, 1), np.uint32)
        native.check(native.lib().sg_verify_queries(be.h, None, tabs, len(flat), status.ctypes.data))
    finally:
        dev.close()
    q0 = 0
    for pr, pi in zip(flat, owners):
        nq = len(pr["iotas"])
        if out[pi][0]:
            bad = np.nonzero(status[q0:q0 + nq])[0]
            if bad.size:
                code = int(status[q0 + bad[0]])
                out[pi] = (False, _REASONS[code & 0xFF].format(code >> 8))
        q0 += nq
    return out


def verify_many(items, opts, be, label=b"lambda_vm_b200/synthetic-multi-table"):
    """Batched verification: [(airs, proof)] or [(airs, proof, label,
    public_terms)] -> [(ok, reason)]; every proof's transcript is replayed on
    the host, then all their queries are checked in one GPU launch."""
    results, preps, idx = [], [], []
    for item in items:
        airs, proof = item[0], item[1]
        lab = item[2] if len(item) > 2 else label
        pub = item[3] if len(item) > 3 else ()
        ok, reason, prep = _replay(airs, proof, opts, lab, pub)
        results.append((ok, reason))
        if ok:
            idx.append(len(results) - 1)
            preps.append(prep)
    for i, r in zip(idx, verify_queries_gpu(preps, be)):
        results[i] = r
    return results


def verify_bytes(airs, blob, opts, label=b"lambda_vm_b200/synthetic-multi-table"):
    from .proof_io import deserialize
    try:
        proof = deserialize(blob)
    except ValueError as e:
        return False, f"malformed proof: {e}"
    return verify(airs, proof, opts, label)
