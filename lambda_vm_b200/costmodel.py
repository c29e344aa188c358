"""Learned cost model of the DFT passes: data, GPU training, tile choice.

The DFT tile width (columns per tile) of every pass is picked at run time
(csrc/ntt.cu). Without a model the context times each compiled width once on
a proxy shape per pass length and scales by the padded column count; that
probe ranks widths unlike the real passes for some shapes. The model here
predicts log(ms) of a pass from its shape and width (features: the C
function sg_pass_features), is trained on the GPU by the library's own MLP
kernels (csrc/mlp.cu) from measured passes (the context's pass log), and once
installed in a context (sg_ctx_set_pass_model) makes the width choice with no
probe launches.

  collect(be)              sweep LDE shapes x pinned widths on the GPU -> records
  train(be, records, ...)  fit the MLP with sg_mlp_train -> parameters
  evaluate(...)            held-out regret of the model and of the probe rule
  install(be, params)      hand the parameters to a context

`python -m lambda_vm_b200.costmodel` on a GPU re-collects the committed
dataset (data/dft_pass_timings.json) and re-trains the committed parameters
(data/pass_model.json) for the GPU it runs on.
"""
import ctypes as C
import hashlib
import json
import math
import os

import numpy as np

from . import native

HERE = os.path.dirname(os.path.abspath(__file__))
DATASET = os.path.join(HERE, "data", "dft_pass_timings.json")
MODEL = os.path.join(HERE, "data", "pass_model.json")
P = 0xFFFFFFFF00000001
SHAPE_KEYS = ("log_len", "tiles", "m", "reps", "inverse", "pre", "post", "canon")


def tile_widths(log_len):
    """Compiled tile widths of a pass length (ntt.cu tile_variants)."""
    if 8 <= log_len <= 10:
        return (4, 8, 16)
    if log_len == 11:
        return (4, 8)
    return ()


def default_width(log_len):
    return 32 if log_len <= 7 else (16 if log_len <= 10 else (8 if log_len == 11 else 4))


def features(rec, cols):
    """Model inputs of the pass `rec` (a dict with SHAPE_KEYS) at tile width `cols`."""
    out = (C.c_float * native.MLP_IN)()
    native.lib().sg_pass_features(rec["log_len"], rec["tiles"], rec["m"], cols, rec["reps"], rec["inverse"],
                                  rec["pre"], rec["post"], rec["canon"], out)
    return np.frombuffer(out, np.float32).copy()


def shape_of(rec):
    return tuple(int(rec[k]) for k in SHAPE_KEYS)


# ---------------------------------------------------------------- data
def _weights(n, g=3):
    ninv = pow(n, P - 2, P)
    w = np.empty(n, np.uint64)
    step = 4096
    gs = [pow(g, i, P) for i in range(step)]
    gstep, base = pow(g, step, P), ninv
    for b in range(0, n, step):
        w[b:b + min(step, n - b)] = [base * x % P for x in gs[:min(step, n - b)]]
        base = base * gstep % P
    return w


def sweep_configs(max_cells=1 << 28):
    """(log_n, m, blowup) of the collection sweep: LDEs whose output has at
    most max_cells words."""
    ms = (1, 2, 3, 4, 6, 8, 9, 12, 16, 20, 24, 32, 40, 48, 64, 100, 128, 200, 256, 300)
    out = []
    for log_n in range(8, 23):
        for m in ms:
            for blowup in (2, 4):
                if (1 << log_n) * m * blowup <= max_cells:
                    out.append((log_n, m, blowup))
    return out


def collect(be, configs=None, repeats=3, seed=5):
    """Time every config's LDE with each compiled tile width pinned, through
    the pass log; returns {"records": [...], "probe": {log_len: {cols: cost}}}.
    Each record is one pass (its shape, width and the median ms of `repeats`)."""
    L = native.lib()
    configs = configs or sweep_configs()
    cols, cost, cnt = (C.c_uint32 * 4)(), (C.c_float * 4)(), C.c_uint32()
    probe = {}
    for log_len in range(8, 12):
        native.check(L.sg_ctx_dft_tuning(be.h, None, log_len, cols, cost, C.byref(cnt)))
        probe[log_len] = {int(cols[i]): float(cost[i]) for i in range(cnt.value)}
    max_in = max((1 << ln) * m for ln, m, _ in configs)
    max_out = max((1 << ln) * m * b for ln, m, b in configs)
    max_n = max(1 << ln for ln, _, _ in configs)
    rng = np.random.default_rng(seed)
    from .device import DeviceBuffer
    dt = DeviceBuffer(max_in * 8, be)
    dw = DeviceBuffer(max_n * 8, be)
    do = DeviceBuffer(max_out * 8, be)
    dt.upload(rng.integers(0, 2**63, size=max_in, dtype=np.uint64))
    weights = {}
    recs = {}
    buf = (native.PassRecord * 64)()
    count = C.c_uint32()
    try:
        for log_n, m, blowup in configs:
            n = 1 << log_n
            if log_n not in weights:
                weights[log_n] = _weights(n)
            dw.upload(weights[log_n])
            lens = {log_n} if log_n <= 12 else {log_n // 2, log_n - log_n // 2}
            widths = sorted({c for ll in lens for c in tile_widths(ll)}) or [0]
            for c in widths:
                for ll in lens:
                    pin = c if c in tile_widths(ll) else 0
                    if tile_widths(ll):
                        native.check(L.sg_ctx_dft_tiles(be.h, ll, pin))
                native.check(L.sg_coset_lde(be.h, None, dt.ptr, n, m, blowup, dw.ptr, do.ptr))  # warm
                native.check(L.sg_stream_sync(be.h, None))
                native.check(L.sg_ctx_pass_log(be.h, 1))
                for _ in range(repeats):
                    native.check(L.sg_coset_lde(be.h, None, dt.ptr, n, m, blowup, dw.ptr, do.ptr))
                native.check(L.sg_ctx_pass_log(be.h, 0))
                native.check(L.sg_ctx_pass_log_read(be.h, buf, 64, C.byref(count)))
                for i in range(count.value):
                    r = buf[i]
                    rec = {k: int(getattr(r, k)) for k in SHAPE_KEYS}
                    key = (shape_of(rec), int(r.cols), (log_n, m, blowup))
                    recs.setdefault(key, (rec, []))[1].append(float(r.ms))
    finally:
        for ll in range(8, 12):
            L.sg_ctx_dft_tiles(be.h, ll, 0)
        for b in (dt, dw, do):
            b.close()
    records = []
    for (shape, cols_, cfg), (rec, ms) in recs.items():
        records.append(dict(rec, cols=cols_, ms=round(float(np.median(ms)), 5), lde=list(cfg)))
    return {"records": records, "probe": {str(k): {str(c): v for c, v in d.items()} for k, d in probe.items()}}


FIELDS = SHAPE_KEYS + ("cols", "ms", "lde_log_n", "lde_m", "lde_blowup")


def save_dataset(data, path=DATASET):
    """Compact JSON: one row of numbers per pass record."""
    rows = [[r[k] for k in SHAPE_KEYS] + [r["cols"], r["ms"]] + list(r["lde"]) for r in data["records"]]
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"fields": list(FIELDS), "rows": rows, "probe": data["probe"]}, f, separators=(",", ":"))


def load_dataset(path=DATASET):
    d = json.load(open(path))
    recs = []
    for row in d["rows"]:
        r = dict(zip(d["fields"], row))
        r["lde"] = [r.pop("lde_log_n"), r.pop("lde_m"), r.pop("lde_blowup")]
        recs.append(r)
    return {"records": recs, "probe": d["probe"]}


# ---------------------------------------------------------------- split, features
def split(records, holdout=0.25):
    """Train / held-out split by LDE config (every pass of a held-out LDE shape
    is held out), by a fixed hash of the config."""
    train, test = [], []
    for r in records:
        h = int(hashlib.sha256(repr(tuple(r["lde"])).encode()).hexdigest()[:8], 16) / 0xFFFFFFFF
        (test if h < holdout else train).append(r)
    return train, test


def design(records):
    X = np.stack([features(r, r["cols"]) for r in records]).astype(np.float32)
    y = np.array([math.log(max(r["ms"], 1e-4)) for r in records], np.float32)
    return X, y


def init_params(seed=0):
    """He-uniform initial weights, zero biases, in the kernels' layout."""
    rng = np.random.default_rng(seed)
    IN, H = native.MLP_IN, native.MLP_HIDDEN
    W1 = rng.uniform(-1, 1, (H, IN)) * math.sqrt(6.0 / IN)
    W2 = rng.uniform(-1, 1, (H, H)) * math.sqrt(6.0 / H)
    w3 = rng.uniform(-1, 1, H) * math.sqrt(6.0 / H)
    p = np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, np.zeros(1)]).astype(np.float32)
    assert p.size == native.MLP_PARAMS
    return p


# ---------------------------------------------------------------- GPU training (library kernels)
def _dev(a, be):
    from .device import DeviceBuffer
    return DeviceBuffer.from_host(np.ascontiguousarray(a, np.float32), be)


def loss_grad(be, X, y, params):
    """One forward + backward pass over the batch on the GPU: (loss, gradient)."""
    dx, dy, dp = _dev(X, be), _dev(y, be), _dev(params, be)
    dg, dl = _dev(np.zeros(native.MLP_PARAMS, np.float32), be), _dev(np.zeros(1, np.float32), be)
    native.check(native.lib().sg_mlp_loss_grad(be.h, None, dx.ptr, dy.ptr, len(y), dp.ptr, dg.ptr, dl.ptr))
    g, l = dg.download(np.float32), dl.download(np.float32)
    for b in (dx, dy, dp, dg, dl):
        b.close()
    return float(l[0]), g


def train(be, X, y, steps=4000, lr=3e-3, seed=0, params=None):
    """Full-batch Adam on the GPU (sg_mlp_train); returns (params, final loss)."""
    p0 = init_params(seed) if params is None else np.asarray(params, np.float32)
    dx, dy, dp = _dev(X, be), _dev(y, be), _dev(p0, be)
    loss = C.c_float()
    native.check(native.lib().sg_mlp_train(be.h, None, dx.ptr, dy.ptr, len(y), dp.ptr, steps, lr, C.byref(loss)))
    p = dp.download(np.float32)
    for b in (dx, dy, dp):
        b.close()
    return p, float(loss.value)


def predict(be, X, params):
    dx, dp = _dev(X, be), _dev(params, be)
    from .device import DeviceBuffer
    do = DeviceBuffer(4 * len(X), be)
    native.check(native.lib().sg_mlp_predict(be.h, None, dx.ptr, len(X), dp.ptr, do.ptr))
    out = do.download(np.float32)
    for b in (dx, dp, do):
        b.close()
    return out


def predict_host(params, X):
    """The same forward pass on the host in float32 (what the tile chooser runs)."""
    IN, H = native.MLP_IN, native.MLP_HIDDEN
    p = np.asarray(params, np.float32)
    o = 0
    W1 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    h1 = np.maximum(X @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h2 @ w3 + b3


# ---------------------------------------------------------------- choices and regret
def probe_pick(probe, log_len, m):
    """The width the timing probe picks (ntt.cu pick_cols without a model)."""
    costs = probe.get(str(log_len)) or probe.get(log_len)
    d = default_width(log_len)
    if not costs:
        return d
    costs = {int(c): float(v) for c, v in costs.items()}
    best_c, best = None, None
    for c, cost in costs.items():
        v = (m + c - 1) // c * c * cost
        if best is None or v < best:
            best, best_c = v, c
    at_def = (m + d - 1) // d * d * costs[d] if d in costs else None
    if at_def is not None and best > 0.97 * at_def:
        return d
    return best_c


def model_pick(params, rec, widths):
    X = np.stack([features(rec, c) for c in widths])
    return widths[int(np.argmin(predict_host(params, X)))]


def evaluate(records, params, probe):
    """Per pass shape with at least two widths measured: the time of the
    width each method picks against the fastest width. Returns sums over the
    shapes (ms) and the mean relative regret of the model, the probe rule and
    the fixed default width."""
    by = {}
    for r in records:
        by.setdefault(shape_of(r), {})[int(r["cols"])] = float(r["ms"])
    tot = {"best": 0.0, "model": 0.0, "probe": 0.0, "default": 0.0}
    reg = {"model": [], "probe": [], "default": []}
    shapes = 0
    for shape, times in by.items():
        if len(times) < 2:
            continue
        rec = dict(zip(SHAPE_KEYS, shape))
        widths = sorted(times)
        best = min(times.values())
        picks = {"model": model_pick(params, rec, widths), "probe": probe_pick(probe, rec["log_len"], rec["m"]),
                 "default": default_width(rec["log_len"])}
        tot["best"] += best
        for k, c in picks.items():
            t = times.get(c, best)
            tot[k] += t
            reg[k].append(t / best - 1.0)
        shapes += 1
    return {"shapes": shapes, "ms": {k: round(v, 4) for k, v in tot.items()},
            "mean_regret": {k: round(float(np.mean(v)), 5) if v else None for k, v in reg.items()}}


def install(be, params):
    """Hand the parameters to the context: its DFT tile widths become the model's choice."""
    p = np.ascontiguousarray(params, np.float32)
    native.check(native.lib().sg_ctx_set_pass_model(be.h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))


def uninstall(be):
    native.check(native.lib().sg_ctx_set_pass_model(be.h, None, 0))


def load_model(path=MODEL):
    d = json.load(open(path))
    return np.array(d["params"], np.float32), d


def main():
    from .device import backend
    be = backend(0)
    data = collect(be)
    save_dataset(data)
    data = load_dataset()
    tr, te = split(data["records"])
    X, y = design(tr)
    params, loss = train(be, X, y)
    ev = evaluate(te, params, data["probe"])
    json.dump({"params": [float(v) for v in params], "train_loss": loss, "train_records": len(tr),
               "heldout": ev, "steps": 4000, "lr": 3e-3, "seed": 0}, open(MODEL, "w"))
    print(json.dumps({"records": len(data["records"]), "train_loss": loss, "heldout": ev}))


if __name__ == "__main__":
    main()
