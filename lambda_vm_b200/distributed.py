"""One proof over several GPUs: tables partitioned across ranks.

The tables of one proof are independent except for one exchange step: after
round 1 every table's 32-byte main root is absorbed, in table order, before
the LogUp challenges are sampled (crypto/stark/src/prover.rs:3458-3490); after
that each table proves on its own transcript fork (prover.rs:3529-3538). So
each rank commits and proves only its share of the tables, the ranks exchange
the roots (32 bytes per table, an all-gather), and rank 0 assembles the
per-table proofs. The proof is the same as the single-GPU prover's.

Tables are assigned heaviest first to the least-loaded rank (longest
processing time first), with a table's weight its LDE cells.
"""
import torch.distributed as dist

from . import field as F
from .ir import device_program, lowered
from .stark import Options, _gen_trace, _u64le, prove_table


def table_weight(air, opts):
    return air.n * opts.blowup * (air.width + 3 * air.aux_width)


def assign_tables(airs, opts, world):
    """Heaviest-first greedy partition: list of table indices per rank."""
    order = sorted(range(len(airs)), key=lambda i: (-table_weight(airs[i], opts), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += table_weight(airs[i], opts)
    return [sorted(p) for p in parts]


def multi_prove_distributed(airs, sources, opts=None, bk=None, group=None,
                            label=b"lambda_vm_b200/synthetic-multi-table"):
    """Prove one multi-table statement across the ranks of `group` (every rank
    calls this with the same arguments and its own backend `bk`). Returns the
    proof dict on rank 0 and None elsewhere."""
    opts = opts or Options()
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    mine = assign_tables(airs, opts, world)[rank]
    B, g = opts.blowup, opts.coset_offset
    # R1 on this rank's tables
    local = {}
    for i in mine:
        tm = _gen_trace(bk, airs[i], sources[i])
        lde = bk.lde(tm, B, bk.domain(airs[i].log_n, B, g).weights)
        tree, root = bk.commit(lde)
        local[i] = (tm, lde, tree, root)
    # the exchange step: every rank learns every table's root
    gathered = [None] * world
    dist.all_gather_object(gathered, {i: v[3] for i, v in local.items()}, group=group)
    roots = {}
    for part in gathered:
        roots.update(part)
    if sorted(roots) != list(range(len(airs))):
        raise RuntimeError("root exchange: missing tables")
    t = bk.transcript(label)
    for i in range(len(airs)):
        t.append_bytes(roots[i])
    challenges = [F.f3(t.sample_ext3()), F.f3(t.sample_ext3())]
    alpha = challenges[1]
    alpha_pows = [(1, 0, 0)]
    for _ in range(max(a.max_alpha for a in airs) - 1):
        alpha_pows.append(F.f3mul(alpha_pows[-1], alpha))
    proofs = {}
    for i in mine:
        ti = t.clone()
        if len(airs) > 1:
            ti.append_bytes(_u64le(i))
        tm, lde, tree, root = local[i]
        p = prove_table(bk, airs[i], lowered(device_program(airs[i])), tm, lde, tree, ti, challenges, alpha_pows, opts)
        p["main_root"] = root
        proofs[i] = p
        bk.free(tm, lde, tree)
    out = [None] * world if rank == 0 else None
    dist.gather_object(proofs, out, dst=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    if rank != 0:
        return None
    allp = {}
    for part in out:
        allp.update(part)
    return {"tables": [allp[i] for i in range(len(airs))], "challenges": challenges}
