"""Several systems advanced together (sfq_group_*) and the tile autotuner (sfq_engine_autotune):
a group block gives every member exactly the block it gets alone, under every lane schedule; the
tuned tiles are valid and reproducible, and any tile choice stays within the mixed tolerances of
the FP64 step."""
import numpy as np
import pytest

from safire_b200 import afqmc as A
from safire_b200 import capi, synthetic

pytestmark = pytest.mark.gpu

BLK = dict(ortho_interval=5, pop_interval=10, equilibration_steps=0, measure_interval=10, relax=0.1, steer=True)

# uneven members: sizes, walker counts and precisions all differ
MEMBERS = [
    (synthetic.SystemSpec(M=48, N=12, Nc=240, decay=48.0, seed=31), 70, capi.PRECISION_MIXED_FP32),
    (synthetic.SystemSpec(M=80, N=20, Nc=400, decay=80.0, seed=32), 131, capi.PRECISION_MIXED),
    (synthetic.SystemSpec(M=64, N=16, Nc=320, decay=64.0, seed=33), 64, capi.PRECISION_FP64),
    (synthetic.SystemSpec(M=112, N=28, Nc=560, decay=112.0, seed=34), 96, capi.PRECISION_MIXED_FP32),
]


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _engines(seed0=100):
    out = []
    for i, (spec, W, prec) in enumerate(MEMBERS):
        out.append(A.AfqmcEngine(synthetic.make_system(spec), W, dt=2e-4, seed=seed0 + i, precision=prec))
    return out


@pytest.mark.parametrize("lanes", [0, 1, 2])
def test_group_block_equals_each_member_alone(lanes):
    grouped, alone = _engines(), _engines()
    E0 = np.array([e.init() for e in grouped])
    for e in alone:
        e.init()
    grp = A.EngineGroup(grouped)
    grp.set_lanes(lanes)
    Eg, st, mg = grp.run_block(20, E0, step0=0, **BLK)
    Eg2, st2, mg2 = grp.run_block(20, Eg, step0=20, **BLK)  # the replayed graph
    assert not st.any() and not st2.any()
    for i, e in enumerate(alone):
        Ea, ma = e.run_block(20, E0[i], step0=0, **BLK)
        Ea2, ma2 = e.run_block(20, Ea, step0=20, **BLK)
        assert Eg[i] == Ea and Eg2[i] == Ea2
        assert len(mg[i]) == len(ma) == 2 and np.array_equal(mg[i], ma) and np.array_equal(mg2[i], ma2)
        S1, p1 = grouped[i].walkers()
        S2, p2 = e.walkers()
        assert np.array_equal(S1, S2)
        for k in ("WEIGHT", "OVLP", "PHASE"):
            assert np.array_equal(p1[k], p2[k])
    # the members stay usable on their own after a group block
    Es, _m = grouped[0].run_block(10, Eg2[0], step0=40, **BLK)
    Ea, _m = alone[0].run_block(10, Eg2[0], step0=40, **BLK)
    assert Es == Ea
    grp.close()
    for e in grouped + alone:
        e.close()


def _int8_engines(seed0=200):
    """INT8X3 members whose products differ in every shape: synthetic CLOSED systems (Taylor tiles of
    64 and 80 orbitals), the reference's Li COLLINEAR and BH GHF NONCOLLINEAR fixtures (tiles of 32)
    and its 34-determinant BH CASCI trial (the force bias from the full G)."""
    from tests.golden_io import engine_system, snapshot
    systems = [(synthetic.make_system(spec), W) for spec, W, _p in MEMBERS]
    systems += [(engine_system(snapshot("li_rohf_collinear")), 40), (engine_system(snapshot("bh_ghf_noncollinear")), 50),
                (engine_system(snapshot("bh_rcasci_uhf_collinear")), 24)]
    return [A.AfqmcEngine(s, W, dt=2e-4, seed=seed0 + i, precision=capi.PRECISION_INT8X3)
            for i, (s, W) in enumerate(systems)]


def test_fused_group_block_equals_each_member_alone():
    """Fused schedule: every stage's int8-slice products of all members (force bias, vHS, P1, Taylor
    terms, the exchange tensor's chunks) run as ONE grouped launch; each member's blocks, its
    measurements and walkers equal its blocks run alone bit for bit, captured and replayed."""
    grouped, alone = _int8_engines(), _int8_engines()
    E0 = np.array([e.init() for e in grouped])
    for e in alone:
        e.init()
    grp = A.EngineGroup(grouped)
    grp.set_fused(True)
    Eg, st, mg = grp.run_block(20, E0, step0=0, **BLK)
    Eg2, st2, mg2 = grp.run_block(20, Eg, step0=20, **BLK)  # the replayed graph
    assert not st.any() and not st2.any()
    for i, e in enumerate(alone):
        Ea, ma = e.run_block(20, E0[i], step0=0, **BLK)
        Ea2, ma2 = e.run_block(20, Ea, step0=20, **BLK)
        assert Eg[i] == Ea and Eg2[i] == Ea2, i
        assert len(mg[i]) == len(ma) == 2 and np.array_equal(mg[i], ma) and np.array_equal(mg2[i], ma2), i
        S1, p1 = grouped[i].walkers()
        S2, p2 = e.walkers()
        assert np.array_equal(S1, S2), i
        for k in ("WEIGHT", "OVLP", "PHASE"):
            assert np.array_equal(p1[k], p2[k]), (i, k)
    # back to lanes: the same members, a block each way again equal
    grp.set_fused(False)
    grp.set_lanes(1)
    Eg3, st3, _m = grp.run_block(10, Eg2, step0=40, **BLK)
    for i, e in enumerate(alone):
        Ea3, _m = e.run_block(10, Eg2[i], step0=40, **BLK)
        assert Eg3[i] == Ea3
    grp.close()
    for e in grouped + alone:
        e.close()


def test_fused_group_refusals():
    es = _engines()[:2]  # split-BF16 members: no int8-slice products to group
    grp = A.EngineGroup(es)
    with pytest.raises(capi.SafireError) as ex:
        grp.set_fused(True)
    assert ex.value.code == 3
    grp.close()
    for e in es:
        e.close()
    es = _int8_engines()[:2]
    grp = A.EngineGroup(es)
    grp.set_fused(True)
    E0 = np.array([e.init() for e in es])
    rps_a = dict(BLK)
    rps_b = dict(BLK, ortho_interval=4)
    grp.block_async(10, E0, **rps_a)
    grp.block_result()
    # one member on another block schedule: refused before anything runs
    with pytest.raises(capi.SafireError) as ex:
        grp.block_async(10, E0, step0=[0, 3], **rps_b)
    assert ex.value.code == 2
    grp.close()
    for e in es:
        e.close()


def test_group_rejects_bad_use():
    es = _engines()[:2]
    with pytest.raises(capi.SafireError):
        A.EngineGroup([es[0], es[0]])
    grp = A.EngineGroup(es)
    with pytest.raises(capi.SafireError):
        grp.set_lanes(-1)
    E0 = np.array([e.init() for e in es])
    grp.block_async(10, E0, **BLK)
    with pytest.raises(capi.SafireError) as ex:
        grp.block_async(10, E0, **BLK)  # the first block's results were not taken
    assert ex.value.code == 2
    grp.block_result()
    grp.close()
    for e in es:
        e.close()


def test_autotune_valid_and_reproducible():
    spec = synthetic.SystemSpec(M=112, N=28, Nc=560, decay=112.0, seed=40)
    s = synthetic.make_system(spec)
    W = 150
    tuned = A.AfqmcEngine(s, W, dt=2e-4, seed=3, precision=capi.PRECISION_MIXED)
    twin = A.AfqmcEngine(s, W, dt=2e-4, seed=3, precision=capi.PRECISION_MIXED)
    E0 = tuned.init()
    twin.init()
    SM0, pr0 = tuned.walkers()
    t = tuned.autotune(repeats=5)
    ch = t.choice()
    assert ch["g_bn"] in (64, 128, 160, 208, 256) and ch["vbias_bn"] in (64, 128, 160, 208, 256)
    assert ch["taylor_half"] in (16, 32, 64, 80, 128) and ch["p1_bn"] in (64, 128, 160, 208, 256)
    assert ch["vbias_ksplit"] >= 1
    for k in range(5):
        assert 0.0 < t.us_tuned[k] <= t.us_builtin[k] * 1.0000001
    # tuning wrote no walker state
    SM1, pr1 = tuned.walkers()
    assert np.array_equal(SM0, SM1) and np.array_equal(pr0["WEIGHT"], pr1["WEIGHT"])
    assert tuned.tiles() == ch
    # the same tiles set on a twin reproduce the tuned engine's block bit for bit
    twin.set_tiles(**ch)
    assert twin.tiles() == ch
    Et, mt = tuned.run_block(20, E0, step0=0, **BLK)
    Ew, mw = twin.run_block(20, E0, step0=0, **BLK)
    assert Et == Ew and np.array_equal(mt, mw)
    assert np.array_equal(tuned.walkers()[0], twin.walkers()[0])
    tuned.close()
    twin.close()


@pytest.mark.parametrize("tiles", [dict(g_bn=64, vbias_bn=256, vhs_bn=64, taylor_half=16, p1_bn=256),
                                   dict(g_bn=208, vbias_bn=64, vhs_bn=160, taylor_half=128, p1_bn=64)])
def test_tile_choices_keep_mixed_accuracy(tiles):
    """Every tile width computes the same products: one mixed step with unusual tiles stays within
    the mixed tolerances of the FP64 step from identical walkers and fields."""
    spec = synthetic.SystemSpec(M=144, N=36, Nc=720, decay=144.0, seed=41)
    s = synthetic.make_system(spec)
    W = 96
    e = A.AfqmcEngine(s, W, dt=2e-4, seed=4, precision=capi.PRECISION_MIXED)
    e64 = A.AfqmcEngine(s, W, dt=2e-4, seed=4, precision=capi.PRECISION_FP64)
    e.set_tiles(**tiles)
    E0 = e64.init()
    e.init()
    SM, pr = e64.walkers()
    e.set_walkers(SM, pr)
    e.propagate(E0, 0)
    e64.propagate(E0, 0)
    S, p = e.walkers()
    S64, p64 = e64.walkers()
    assert _rel(S, S64) < 2e-4
    assert _rel(p["OVLP"], p64["OVLP"]) < 2e-3
    e.close()
    e64.close()


def test_int8_taylor_tiles_tuned_and_exact():
    """INT8X3: the Taylor term's orbitals per tile (32, 64, 80) change only the tiling of an exact
    integer product, so blocks at every width are equal bit for bit; the tuner picks one of them
    from timings on the engine's operands and writes no walker state."""
    spec = synthetic.SystemSpec(M=144, N=36, Nc=720, decay=144.0, seed=43)
    s = synthetic.make_system(spec)
    W = 96
    out = []
    for h in (32, 64, 80):
        e = A.AfqmcEngine(s, W, dt=2e-4, seed=6, precision=capi.PRECISION_INT8X3)
        E0 = e.init()
        e.set_tiles(taylor_half=h)
        assert e.tiles()["taylor_half"] == h
        out.append((e.run_block(10, E0, step0=0, **BLK), e.walkers()))
        e.close()
    for (Eb, mb), (S, p) in out[1:]:
        assert Eb == out[0][0][0] and np.array_equal(mb, out[0][0][1])
        assert np.array_equal(S, out[0][1][0]) and np.array_equal(p["WEIGHT"], out[0][1][1]["WEIGHT"])
    e = A.AfqmcEngine(s, W, dt=2e-4, seed=6, precision=capi.PRECISION_INT8X3)
    E0 = e.init()
    SM0, pr0 = e.walkers()
    t = e.autotune(repeats=5)
    ch = t.choice()
    assert ch["taylor_half"] in (32, 64, 80) and ch["g_bn"] == 0
    assert 0.0 < t.us_tuned[3] <= t.us_builtin[3] * 1.0000001
    SM1, pr1 = e.walkers()
    assert np.array_equal(SM0, SM1) and np.array_equal(pr0["WEIGHT"], pr1["WEIGHT"])
    assert e.run_block(10, E0, step0=0, **BLK)[0] == out[0][0][0]
    with pytest.raises(capi.SafireError) as ex:
        e.set_tiles(taylor_half=48)
    assert ex.value.code == 2
    with pytest.raises(capi.SafireError) as ex:
        e.set_tiles(g_bn=64)
    assert ex.value.code == 2
    e.close()


def test_tiles_rejected():
    s = synthetic.make_system(synthetic.SystemSpec(M=48, N=12, Nc=240, decay=48.0, seed=42))
    e = A.AfqmcEngine(s, 32, dt=2e-4, seed=1, precision=capi.PRECISION_MIXED_FP32)
    with pytest.raises(capi.SafireError) as ex:
        e.set_tiles(p1_bn=208)  # not built for 3 planes
    assert ex.value.code == 2
    with pytest.raises(capi.SafireError) as ex:
        e.set_tiles(taylor_half=48)
    assert ex.value.code == 2
    e.close()
    e64 = A.AfqmcEngine(s, 32, dt=2e-4, seed=1, precision=capi.PRECISION_FP64)
    with pytest.raises(capi.SafireError) as ex:
        e64.autotune()
    assert ex.value.code == 3
    e64.close()
