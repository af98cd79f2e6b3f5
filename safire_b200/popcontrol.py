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
    SM, props = population_control(dist, SM, props, r, group)   # collective; r used on the root

Within one rank the copies fill the slots of walkers that leave, in the order swap_walkers_async
fills them (population_control.hpp:143-209), so one rank reproduces the single-rank comb exactly.
"""
import numpy as np

WEIGHT = 0  # property column of the weights


def comb(weights, r, num_target):
    """The comb over |w| with the uniform r (population_control.hpp:34-65): offspring per walker."""
    w = np.asarray(weights, dtype=np.float64)
    cum = np.cumsum(w)  # std::partial_sum, sequential
    total = float(cum[-1])
    if not total > 1e-6:
        raise RuntimeError(f"The total walker weight collapsed to {total}.")
    last = len(w) - 1
    while w[last] <= 0.0:
        last -= 1
    off = np.zeros(len(w), dtype=np.int64)
    iw = ic = 0
    while ic < num_target:
        if (ic + r) * total / num_target < cum[iw] or iw == last:
            off[iw] += 1
            ic += 1
        else:
            iw += 1
    return off


def plan_walker_exchange(offspring, counts):
    """(src rank, local walker, dst rank, copies) transfers realising offspring (rank-major over the
    global population, rank r holding counts[r] walkers): ranks with excess export their walkers with
    the most copies first, filling the ranks with a deficit in rank order (population_control.hpp:73-133)."""
    offspring = np.asarray(offspring, dtype=np.int64)
    counts = [int(c) for c in counts]
    if offspring.size != sum(counts) or int(offspring.sum()) != sum(counts):
        raise ValueError("plan_walker_exchange: offspring does not match or preserve the population")
    exports, deficits = [], []
    first = 0
    for r, nw in enumerate(counts):
        local = offspring[first:first + nw]
        excess = int(local.sum()) - nw
        if excess < 0:
            deficits.append([r, -excess])
        if excess > 0:
            order = sorted(range(nw), key=lambda i: -int(local[i]))  # stable: ties keep index order
            k = 0
            while excess > 0:
                m = min(int(local[order[k]]), excess)
                exports.append([r, order[k], m])
                excess -= m
                k += 1
        first += nw
    plan, d = [], 0
    for src, walker, copies in exports:
        while copies > 0:
            n = min(copies, deficits[d][1])
            plan.append((src, walker, deficits[d][0], n))
            copies -= n
            deficits[d][1] -= n
            if deficits[d][1] == 0:
                d += 1
    return plan


def local_moves(offspring, counts, rank):
    """This rank's part of swap_walkers_async (population_control.hpp:143-209): the plan, the sends
    (local walker, dst), the receives (slot, src, copies) in plan order, and the local copies
    (src slot, dst slot) to make after the receives, in the order the reference makes them."""
    plan = plan_walker_exchange(offspring, counts)
    nw = counts[rank]
    first = sum(counts[:rank])
    keep = [int(k) for k in np.asarray(offspring)[first:first + nw]]
    for src, walker, dst, n in plan:
        if src == rank:
            keep[walker] -= n
    free = [i for i in range(nw) if keep[i] == 0]
    nxt = 0
    sends, recvs, arrivals = [], [], []
    for src, walker, dst, n in plan:
        if src == rank:
            sends.append((walker, dst))
        elif dst == rank:
            slot = free[nxt]
            nxt += 1
            recvs.append((slot, src))
            arrivals.append((slot, n))
    copies = []
    for i in range(nw):
        for _ in range(1, keep[i]):
            copies.append((i, free[nxt]))
            nxt += 1
    for slot, n in arrivals:
        for _ in range(1, n):
            copies.append((slot, free[nxt]))
            nxt += 1
    if nxt != len(free):
        raise RuntimeError(f"swap_walkers_async: {len(free) - nxt} slots left unfilled")
    return plan, sends, recvs, copies


def population_control(dist, SM, props, r, group=None):
    """The collective population control on this rank's walker table (SM (nw, rows, cols) complex,
    props (8, nw) complex); r is the root's comb uniform (ignored elsewhere).  Returns the new table:
    walkers copied and exchanged along the plan, weights w / |w|.  With dist None: one rank."""
    import torch
    SM = np.array(SM, dtype=np.complex128)
    props = np.array(props, dtype=np.complex128)
    nw = SM.shape[0]
    rank = dist.get_rank(group) if dist else 0
    size = dist.get_world_size(group) if dist else 1
    if dist:
        cnt = [torch.zeros(1, dtype=torch.int64) for _ in range(size)]
        dist.all_gather(cnt, torch.tensor([nw], dtype=torch.int64), group=group)
        counts = [int(c.item()) for c in cnt]
    else:
        counts = [nw]
    w = np.abs(props[WEIGHT])
    if dist:
        mx = max(counts)
        buf = torch.zeros(mx, dtype=torch.float64)
        buf[:nw] = torch.from_numpy(w)
        allw = [torch.zeros(mx, dtype=torch.float64) for _ in range(size)]
        dist.all_gather(allw, buf, group=group)
        weights = np.concatenate([a.numpy()[:c] for a, c in zip(allw, counts)])
    else:
        weights = w
    off = torch.zeros(sum(counts), dtype=torch.int64)
    if rank == 0:
        off = torch.from_numpy(comb(weights, r, sum(counts)))
    if dist:
        dist.broadcast(off, 0, group=group)
    offspring = off.numpy()
    _, sends, recvs, copies = local_moves(offspring, counts, rank)
    sm_elems = int(np.prod(SM.shape[1:]))  # a rank may hold no walkers
    row = lambda i: torch.from_numpy(np.concatenate([SM[i].reshape(-1), props[:, i]]).view(np.float64))
    # a rank either sends or receives; both ends post in plan order (MPI's non-overtaking rule there)
    for walker, dst in sends:
        dist.send(row(walker).contiguous(), dst, group=group)
    for slot, src in recvs:
        t = torch.empty(2 * (sm_elems + props.shape[0]), dtype=torch.float64)
        dist.recv(t, src, group=group)
        v = t.numpy().view(np.complex128)
        SM[slot] = v[:sm_elems].reshape(SM.shape[1:])
        props[:, slot] = v[sm_elems:]
    for src, dst in copies:
        SM[dst] = SM[src]
        props[:, dst] = props[:, src]
    wt = props[WEIGHT]
    props[WEIGHT] = wt / np.abs(wt)
    return SM, props


def engine_population_control(dist, engine, r, group=None):
    """population_control for an AfqmcEngine whose walkers are this rank's share of the population:
    the engine's walker table goes through the collective comb and exchange and back (set_walkers)."""
    SM, pr = engine.walkers()
    from . import capi
    props = np.stack([pr[k] for k in capi.PROPS])
    SM, props = population_control(dist, SM, props, r, group)
    engine.set_walkers(SM, {k: props[i] for i, k in enumerate(capi.PROPS)})
