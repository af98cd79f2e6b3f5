"""Population control over walkers sharded across ranks (one process per GPU).

The reference's population_control (src/AFQMC/Walkers/population_control.hpp:34-255) is collective
over the ranks: the ranks' |w| are gathered to the root, one comb over the whole population draws
the offspring, the root broadcasts them, and the walkers move between ranks along a deterministic
plan (plan_walker_exchange) that every rank computes, each rank ending with its own target count.
Here the same steps run over torch.distributed (gloo on CPU, NCCL on GPUs) on walker tables: per
rank the Slater matrices SM (nw, rows, cols) and the property columns props (8, nw) -- what
AfqmcEngine.walkers() returns and set_walkers() takes.

    offspring = comb(weights, r, ntot)                # the root's comb (population_control.hpp:34-65)
    plan = plan_walker_exchange(offspring, counts)    # population_control.hpp:73-133
    sends, recvs, copies = local_moves(offspring, counts, rank)   # population_control.hpp:143-209
    SM, props = population_control(dist, SM, props, r, group)   # collective; r used on the root

The comb, the plan and each rank's moves are native host code behind the C ABI (sfq_comb_host,
sfq_plan_walker_exchange, sfq_walker_moves), which needs no device; the data movement runs over
torch.distributed.  Within one rank the copies fill the slots of walkers that leave, in the order
swap_walkers_async fills them (population_control.hpp:143-209), so one rank reproduces the
single-rank comb exactly.

engine_population_control runs the same steps on an engine's resident walker table without taking
it off the device: only the |w| column (8 bytes per walker) goes to the host for the gather and the
comb; the walkers that leave are packed on the device into rows (sfq_engine_pack_walkers), the rows
cross ranks as device tensors (NCCL send/recv; through the host under gloo), arrive in a device
buffer and are scattered into the free slots (sfq_engine_unpack_walkers), and the local copies and
the weight normalisation run as one device call (sfq_engine_copy_walkers).
"""
import numpy as np

from . import capi

WEIGHT = 0  # property column of the weights


def _i32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


def _cell():
    """A one-int output of the C ABI."""
    return np.zeros(1, dtype=np.int32)


def _population(offspring, counts):
    """offspring and counts as int32 arrays, checked against each other (the C ABI cannot see the
    length of offspring, which must be sum(counts))."""
    off, cnt = _i32(offspring).ravel(), _i32(counts).ravel()
    if cnt.size == 0 or off.size != int(cnt.sum()):
        raise capi.SafireError(2, f"{off.size} offspring entries for ranks holding {cnt.tolist()} walkers")
    return off, cnt


def comb(weights, r, num_target):
    """The comb over |w| with the uniform r (population_control.hpp:34-65): offspring per walker.
    Native host code (sfq_comb_host); raises SafireError WEIGHT_COLLAPSE when the total weight
    collapses."""
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
    off = np.zeros(w.size, dtype=np.int32)
    capi.check(capi.lib().sfq_comb_host(capi.ptr(w), float(r), w.size, int(num_target), capi.ptr(off)))
    return off.astype(np.int64)


def plan_walker_exchange(offspring, counts):
    """(src rank, local walker, dst rank, copies) transfers realising offspring (rank-major over the
    global population, rank r holding counts[r] walkers): ranks with excess export their walkers with
    the most copies first, filling the ranks with a deficit in rank order (population_control.hpp:73-133).
    Native host code (sfq_plan_walker_exchange)."""
    off, cnt = _population(offspring, counts)
    cap = int(cnt.sum()) + cnt.size
    out = np.zeros((cap, 4), dtype=np.int32)
    n = _cell()
    capi.check(capi.lib().sfq_plan_walker_exchange(capi.ptr(off), capi.ptr(cnt), cnt.size, capi.ptr(out), cap,
                                                   capi.ptr(n)))
    return [tuple(int(v) for v in row) for row in out[:int(n[0])]]


def local_moves(offspring, counts, rank):
    """This rank's part of swap_walkers_async (population_control.hpp:143-209): the sends (local
    walker, dst) and receives (slot, src) in plan order, and the local copies (src slot, dst slot) to
    make after the receives, in the order the reference makes them.  Native host code (sfq_walker_moves)."""
    off, cnt = _population(offspring, counts)
    if not 0 <= rank < cnt.size:
        raise capi.SafireError(2, f"rank {rank} of {cnt.size}")
    nw = int(cnt[rank])
    sends = np.zeros((nw + cnt.size, 2), dtype=np.int32)
    recvs = np.zeros((max(nw, 1), 2), dtype=np.int32)
    copies = np.zeros((max(nw, 1), 2), dtype=np.int32)
    ns, nr, nc = _cell(), _cell(), _cell()
    capi.check(capi.lib().sfq_walker_moves(capi.ptr(off), capi.ptr(cnt), cnt.size, int(rank), capi.ptr(sends),
                                           len(sends), capi.ptr(ns), capi.ptr(recvs), len(recvs), capi.ptr(nr),
                                           capi.ptr(copies), len(copies), capi.ptr(nc)))
    pairs = lambda a, n: [(int(x), int(y)) for x, y in a[:int(n[0])]]
    return pairs(sends, ns), pairs(recvs, nr), pairs(copies, nc)


def comm_device(dist, group=None):
    """The device a collective of this group takes its tensors on: the current CUDA device for
    NCCL (which moves only device memory), the host otherwise (gloo)."""
    import torch
    if dist is not None and dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def global_offspring(dist, w, r, group=None):
    """The collective part of population_control (population_control.hpp:219-236): the ranks' walker
    counts and |w| are gathered, the root combs the whole population with its uniform r, and every
    rank receives the offspring.  w: this rank's |w| (host).  Returns (offspring, counts, rank)."""
    import torch
    w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
    nw = w.size
    rank = dist.get_rank(group) if dist else 0
    size = dist.get_world_size(group) if dist else 1
    dev = comm_device(dist, group)
    if dist:
        cnt = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(size)]
        dist.all_gather(cnt, torch.tensor([nw], dtype=torch.int64, device=dev), group=group)
        counts = [int(c.item()) for c in cnt]
        mx = max(counts)
        buf = torch.zeros(mx, dtype=torch.float64)
        buf[:nw] = torch.from_numpy(w)
        allw = [torch.zeros(mx, dtype=torch.float64, device=dev) for _ in range(size)]
        dist.all_gather(allw, buf.to(dev), group=group)
        weights = np.concatenate([a.cpu().numpy()[:c] for a, c in zip(allw, counts)])
    else:
        counts = [nw]
        weights = w
    off = torch.zeros(sum(counts), dtype=torch.int64)
    if rank == 0:
        off = torch.from_numpy(comb(weights, r, sum(counts)))
    if dist:
        off = off.to(dev)
        dist.broadcast(off, 0, group=group)
    return off.cpu().numpy(), counts, rank


def population_control(dist, SM, props, r, group=None):
    """The collective population control on this rank's walker table (SM (nw, rows, cols) complex,
    props (8, nw) complex, host arrays); r is the root's comb uniform (ignored elsewhere).  Returns
    the new table: walkers copied and exchanged along the plan, weights w / |w|.  With dist None:
    one rank."""
    import torch
    SM = np.array(SM, dtype=np.complex128)
    props = np.array(props, dtype=np.complex128)
    dev = comm_device(dist, group)
    offspring, counts, rank = global_offspring(dist, np.abs(props[WEIGHT]), r, group)
    sends, recvs, copies = local_moves(offspring, counts, rank)
    sm_elems = int(np.prod(SM.shape[1:]))  # a rank may hold no walkers
    row = lambda i: torch.from_numpy(np.concatenate([SM[i].reshape(-1), props[:, i]]).view(np.float64)).to(dev)
    # a rank either sends or receives; both ends post in plan order (MPI's non-overtaking rule there)
    for walker, dst in sends:
        dist.send(row(walker).contiguous(), dst, group=group)
    for slot, src in recvs:
        t = torch.empty(2 * (sm_elems + props.shape[0]), dtype=torch.float64, device=dev)
        dist.recv(t, src, group=group)
        v = t.cpu().numpy().view(np.complex128)
        SM[slot] = v[:sm_elems].reshape(SM.shape[1:])
        props[:, slot] = v[sm_elems:]
    for src, dst in copies:
        SM[dst] = SM[src]
        props[:, dst] = props[:, src]
    wt = props[WEIGHT]
    props[WEIGHT] = wt / np.abs(wt)
    return SM, props


def engine_population_control(dist, engine, r, group=None):
    """population_control for an engine whose walkers are this rank's share of the population, with
    the walker table kept on the engine's device.

    Engine interface: properties() (the property columns, host), and the row calls of the walker
    exchange -- exchange_device (where its rows live), walker_row_elems(), pack_walkers(slots, rows),
    unpack_walkers(slots, rows), copy_walkers(pairs, normalize) -- as AfqmcEngine has them over
    sfq_engine_pack_walkers / unpack_walkers / copy_walkers.  Rows are float64 tensors (n, 2 *
    walker_row_elems()) on exchange_device: a walker's Slater matrix then its 8 property values.

    Only the Slater matrices and the property columns travel.  An engine that keeps back-propagation
    history (enable_back_propagation) also holds per-walker field rings, weight factors and anchored
    walkers, which the reference moves with the walker (copy_walker, population_control.hpp:243-247);
    those would stay behind here and pair each walker with another walker's history, so such an
    engine is refused."""
    if getattr(engine, "nbp", 0) > 0:
        raise capi.SafireError(3, "sharded population control does not move back-propagation history; "
                                  "run back propagation on one rank (engine.population_control)")
    import torch
    pr = engine.properties()
    offspring, counts, rank = global_offspring(dist, np.abs(np.asarray(pr["WEIGHT"])), r, group)
    sends, recvs, copies = local_moves(offspring, counts, rank)
    edev = engine.exchange_device
    cdev = comm_device(dist, group)
    width = 2 * int(engine.walker_row_elems())
    # a rank either sends or receives; both ends post in plan order (MPI's non-overtaking rule there)
    if sends:
        rows = torch.empty((len(sends), width), dtype=torch.float64, device=edev)
        engine.pack_walkers([w for w, _ in sends], rows)
        for i, (_, dst) in enumerate(sends):
            dist.send(rows[i] if cdev == edev else rows[i].to(cdev), dst, group=group)
    if recvs:
        rows = torch.empty((len(recvs), width), dtype=torch.float64, device=edev)
        for i, (_, src) in enumerate(recvs):
            if cdev == edev:
                dist.recv(rows[i], src, group=group)
            else:
                t = torch.empty(width, dtype=torch.float64, device=cdev)
                dist.recv(t, src, group=group)
                rows[i].copy_(t)
        if edev.type == "cuda":
            torch.cuda.current_stream(edev).synchronize()  # the receives land before the engine stream reads
        engine.unpack_walkers([slot for slot, _ in recvs], rows)
    if sends and edev.type == "cuda":
        torch.cuda.current_stream(edev).synchronize()  # the sends have read their rows
    engine.copy_walkers(copies, normalize=True)
