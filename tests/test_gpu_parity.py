"""CUDA path vs the FP64 oracle and the reference's known answers, through the C ABI.

Tolerances: the reference KATs are compared with the reference's own utils::Approx (1e-8);
everything against the oracle uses the north-star FP64 bar, 1e-10 relative (max-norm),
except integer/index results (comb offspring, copy plans) which must be bit-exact.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from golden_io import sdet_kats  # noqa: E402
from oracle import afqmc_oracle as O  # noqa: E402
from oracle import philox  # noqa: E402
from safire_b200 import afqmc as A  # noqa: E402
from safire_b200 import synthetic  # noqa: E402

REL = 1e-10


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / den)


def kat(a, b, tol=1e-8):
    """utils::Approx semantics (atol = rtol = 1e-8, tests/test_common.hpp:383-444)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b))) <= tol * max(1.0, float(np.max(np.abs(b))))


def cu(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def kats():
    return sdet_kats()


def _batch(m, nw=5):
    return np.broadcast_to(m, (nw,) + m.shape).copy()


# ---------------------------------------------------------------- reference KATs (1e-8)
def test_kat_log_overlap(kats):
    ov = A.Log_Overlap(cu(kats["m_a"]), cu(_batch(kats["m_b"])))
    assert kat(host(ov), np.full(5, np.log(kats["ov_base_log_of"])))
    ov2 = A.Log_Overlap(cu(kats["m_a"][:2, :3]), cu(_batch(kats["m_b"])[:, :3, :2]))
    assert kat(host(ov2), np.full(5, np.log(kats["ov2_base_log_of"])))


def test_kat_mixed_density_matrix(kats):
    Am, Bm = cu(kats["m_a"]), cu(_batch(kats["m_b"]))
    G, ov = A.MixedDensityMatrix(Am, Bm, compact=False)
    assert kat(host(G), _batch(kats["v_ref"]))
    assert kat(host(ov), np.full(5, np.log(kats["ov_base_log_of"])))
    Gc, _ = A.MixedDensityMatrix(Am, Bm, compact=True)
    assert kat(host(Gc), _batch(kats["vc_ref"]))
    G2, _ = A.MixedDensityMatrix(cu(kats["m_a"][:2, :3]), cu(_batch(kats["m_b"])[:, :3, :2]), compact=False)
    assert kat(host(G2), _batch(kats["v_ref_2"]))
    Gc2, _ = A.MixedDensityMatrix(cu(kats["m_a"][:2, :3]), cu(_batch(kats["m_b"])[:, :3, :2]), compact=True)
    assert kat(host(Gc2), _batch(kats["vc_ref_2"]))


def test_kat_inverse_logdet(kats):
    inv, ld = A.inverse_logdet(cu(_batch(kats["inv_m_a"])))
    assert kat(host(inv), _batch(kats["inv_ref"]))
    assert kat(host(ld), np.full(5, kats["logdetA_ref"]))
    inv, ld = A.inverse_logdet(cu(_batch(kats["ma_lu"])))
    assert kat(host(inv) @ kats["mb_lu"], _batch(kats["xv_ref"]))
    assert kat(host(ld), np.full(5, kats["ovlp_lu_ref"]))


def test_kat_orthogonalize(kats):
    Q = A.orthogonalize(cu(_batch(kats["m_b"])))
    Qh = host(Q)
    ov = O.log_overlap(np.conj(Qh[0].T), Qh)
    assert np.max(np.abs(ov)) < 1e-12
    Qo, _ = O.orthogonalize(_batch(kats["m_b"]))
    assert rel(Qh, Qo) < REL


@pytest.mark.parametrize("N", [40, 100])
def test_inverse_logdet_with_tied_pivots(N):
    """Entries of modulus |re| + |im| = 1 (+-1, +-i): every pivot search starts among exactly tied
    candidates, which zgetrf resolves by the first in its row order; the inverse and log det against
    the oracle's LAPACK factorization."""
    rng = np.random.default_rng(N)
    T = rng.choice(np.array([1, -1, 1j, -1j]), size=(4, N, N))
    assert all(abs(np.linalg.det(t)) > 1e-6 for t in T)
    inv, ld = A.inverse_logdet(cu(T))
    io, lo = O.inverse_logdet(T)
    assert rel(host(inv), io) < 1e-9
    assert np.max(np.abs(host(ld) - lo)) < 1e-9 * np.max(np.abs(lo))


def test_singular_overlap_zero_inverse():
    T = np.zeros((2, 3, 3), np.complex128)
    T[:, 0, 0] = 1.0
    inv, ld = A.inverse_logdet(cu(T))
    assert np.all(host(inv) == 0)
    assert np.all(host(ld).real < -700)


# ---------------------------------------------------------------- operations vs oracle
@pytest.fixture(scope="module")
def sysmed():
    s = synthetic.make_system(synthetic.SystemSpec(M=40, N=10, Nc=120, decay=40.0, seed=5))
    return s, O.Hamiltonian(s.hcore, s.Likn, s.PsiT)


def _walkers(s, W, seed=1, amp=0.3):
    rng = np.random.default_rng(seed)
    return s.initial_walkers(W) + amp * (rng.normal(size=(W, s.M, s.N)) + 1j * rng.normal(size=(W, s.M, s.N)))


@pytest.mark.parametrize("complex_trial", [False, True])
def test_density_and_overlap(sysmed, complex_trial):
    s, ham = sysmed
    Wk = _walkers(s, 13)
    PsiT = ham.PsiT.copy()
    if complex_trial:
        PsiT = PsiT * np.exp(1j * np.linspace(0, 1, s.M))[None, :]
    Go, ovo = O.mixed_density_matrix(PsiT, Wk)
    Ad = cu(PsiT) if complex_trial else cu(PsiT.real.copy())
    G, ov = A.MixedDensityMatrix(Ad, cu(Wk))
    assert rel(host(G), Go) < REL
    assert rel(host(ov), ovo) < REL
    ov2 = A.Log_Overlap(Ad, cu(Wk))
    assert rel(host(ov2), O.log_overlap(PsiT, Wk)) < REL


def test_vbias_vhs_energy(sysmed):
    s, ham = sysmed
    Wk = _walkers(s, 9, seed=3)
    G, _ = O.mixed_density_matrix(ham.PsiT, Wk)
    dt = 0.01
    vb = A.vbias(cu(G), cu(ham.Lnak.real.copy()), dt)
    assert rel(host(vb), ham.vbias(G, dt)) < REL
    vb_c = A.vbias(cu(G), cu(ham.Lnak), dt)
    assert rel(host(vb_c), ham.vbias(G, dt)) < REL
    rng = np.random.default_rng(4)
    X = rng.normal(size=(9, s.Nc)) + 1j * rng.normal(size=(9, s.Nc))
    V = A.vHS(cu(s.Likn), cu(X), dt)
    assert rel(host(V), ham.vHS(X, dt)) < REL
    E = A.energy(cu(G), cu(ham.haj), cu(ham.Lnak.real.copy()), E0=0.7)
    ham.E0 = 0.7
    Eo = ham.energy(G)
    ham.E0 = 0.0
    assert rel(host(E), Eo) < REL


@pytest.mark.parametrize("injected", [True, False])
def test_assemble_x(sysmed, injected):
    s, ham = sysmed
    rng = np.random.default_rng(6)
    W = 7
    vb = rng.normal(size=(W, s.Nc)) + 1j * rng.normal(size=(W, s.Nc))
    vb[0, 0] = 80 + 10j  # beyond vbias_bound: clamped
    vmf = rng.normal(size=s.Nc)
    vmf[3] = -70.0
    seed, step = 11, 123456789012
    u = philox.uniforms(seed, philox.STREAM_FIELDS, step, W, s.Nc)
    Xo, HWo = O.assemble_X(vb, vmf, u, 50.0)
    mfo = O.meanfield_factor(Xo, vmf)
    X, hw, mf = A.assemble_X(cu(vb), cu(vmf), uniforms=cu(u) if injected else None, seed=seed, step=step)
    assert rel(host(X), Xo) < REL
    assert rel(host(hw), HWo) < REL
    assert rel(host(mf), mfo) < REL


def test_propagate_and_orthogonalize(sysmed):
    s, ham = sysmed
    W = 6
    Wk = _walkers(s, W, seed=8, amp=0.1)
    prop = O.Propagator(ham, 0.01)
    rng = np.random.default_rng(9)
    X = rng.normal(size=(W, s.Nc)) + 0.2j * rng.normal(size=(W, s.Nc))
    V = ham.vHS(X, 0.01)
    out = A.Propagate(cu(Wk), cu(prop.P1.real.copy()), cu(V), 6)
    ref = O.propagate(Wk, prop.P1, V, 6)
    assert rel(host(out), ref) < REL
    out_c = A.Propagate(cu(Wk), cu(prop.P1), cu(V), 6)
    assert rel(host(out_c), ref) < REL
    Q = A.orthogonalize(cu(ref))
    Qo, _ = O.orthogonalize(ref)
    assert rel(host(Q), Qo) < REL


def test_comb_bit_exact():
    rng = np.random.default_rng(10)
    for trial in range(30):
        n = int(rng.integers(2, 3000))
        w = rng.exponential(size=n)
        w[rng.integers(0, n, max(1, n // 7))] = 0.0
        if trial % 5 == 0:
            w[-3:] = 0.0  # the last teeth land on the last walker with weight
        r = float(rng.uniform())
        off = host(A.comb(cu(w), r))
        assert np.array_equal(off, O.comb(w, r, n))
        # the host comb a sharded run's root uses draws the same offspring
        from safire_b200 import popcontrol
        assert np.array_equal(popcontrol.comb(w, r, n), off)


def test_comb_weight_collapse():
    from safire_b200.capi import SafireError
    with pytest.raises(SafireError, match="WEIGHT_COLLAPSE"):
        A.comb(cu(np.zeros(8)), 0.5)


# ---------------------------------------------------------------- resident engine vs oracle
def _engine_pair(spec, W, dt=0.005, seed=0):
    s = synthetic.make_system(spec)
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    eng = A.AfqmcEngine(s, W, dt=dt, seed=seed)
    prop = O.Propagator(ham, dt, seed=seed)
    wo = O.Walkers(s.initial_walkers(W))
    return s, ham, eng, prop, wo


def test_engine_setup_tensors():
    s, ham, eng, prop, wo = _engine_pair(synthetic.CFG_SMALL, 4)
    M, N, Nc = s.M, s.N, s.Nc
    assert rel(eng.fetch("Lnak", (Nc, N, M), np.float64), ham.Lnak.real) < REL
    assert rel(eng.fetch("haj", (N, M), np.complex128), ham.haj) < REL
    assert rel(eng.fetch("v0", (M, M), np.float64), ham.v0) < REL
    assert rel(eng.fetch("vmf", (Nc,), np.float64), prop.vmf.real) < REL
    assert rel(eng.fetch("P1", (M, M), np.float64), prop.P1.real) < REL
    eng.close()


def test_engine_energy_and_step():
    s, ham, eng, prop, wo = _engine_pair(synthetic.CFG_SMALL, 16)
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    assert abs(Esh - Esh_o) < REL * abs(Esh_o)
    SM, pr = eng.walkers()
    assert rel(pr["E1_"], wo.e1) < REL and rel(pr["EXX_"], wo.exx) < REL and rel(pr["EJ_"], wo.ej) < REL
    for step in range(3):
        dbg = prop.propagate(wo, Esh_o, step)
        eng.propagate(Esh, step)
        SM, pr = eng.walkers()
        assert rel(eng.fetch("X", (16, s.Nc), np.complex128), dbg["X"]) < REL
        assert rel(SM, wo.SM) < REL
        for k, f in (("WEIGHT", "weight"), ("PHASE", "phase"), ("PSEUDO_ELOC_", "pseudo_eloc"), ("OVLP", "ovlp")):
            assert rel(pr[k], getattr(wo, f)) < REL, k
    eng.orthogonalize()
    prop.orthogonalize(wo)
    SM, pr = eng.walkers()
    assert rel(SM, wo.SM) < REL
    assert rel(pr["OVLP"], wo.ovlp) < REL
    eng.close()


def test_engine_population_control_bit_exact():
    s, ham, eng, prop, wo = _engine_pair(synthetic.CFG_SMALL, 24)
    Esh = eng.init()
    O.init_walkers(ham, wo)
    for step in range(4):
        eng.propagate(Esh, step)
    SM, pr = eng.walkers()
    # hand the engine's own state to the oracle so the comb sees identical weights
    wo.SM = SM.copy()
    for k, f in (("WEIGHT", "weight"), ("PHASE", "phase"), ("PSEUDO_ELOC_", "pseudo_eloc"), ("E1_", "e1"),
                 ("EXX_", "exx"), ("EJ_", "ej"), ("OVLP", "ovlp"), ("THETA", "theta")):
        setattr(wo, f, pr[k].copy())
    # make the comb interesting: spread the weights
    # real positive weights, so |w| is exact on both sides
    w = (np.abs(pr["WEIGHT"]) * np.linspace(0.1, 3.0, 24)).astype(np.complex128)
    w[5] = 0.0
    pr["WEIGHT"] = w
    wo.weight = w.copy()
    eng.set_walkers(props=pr)
    call = 77
    eng.population_control(call)
    O.population_control(wo, philox.comb_uniform(0, call))
    SM2, pr2 = eng.walkers()
    assert np.array_equal(SM2, wo.SM)
    assert np.array_equal(pr2["PSEUDO_ELOC_"], wo.pseudo_eloc)
    assert rel(pr2["WEIGHT"], wo.weight) < 1e-15
    eng.close()


def test_engine_full_run_small():
    """The small configuration end to end: 200 steps, ortho every 5, comb every 20."""
    s, ham, eng, prop, wo = _engine_pair(synthetic.CFG_SMALL, 32)
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    Esh_o, meas_o = O.run(ham, wo, prop, 200, Esh_o, ortho_interval=5, pop_interval=20)
    Esh, meas = eng.run(200, Esh, ortho_interval=5, pop_interval=20)
    assert abs(Esh - Esh_o) < 1e-9 * abs(Esh_o)
    assert len(meas) == len(meas_o)
    for (step, mo), m in zip(meas_o, meas):
        assert abs(complex(m[0], m[1]) - mo["Energy"]) < 1e-9 * abs(mo["Energy"])
    SM, pr = eng.walkers()
    assert rel(pr["WEIGHT"], wo.weight) < 1e-9
    assert rel(SM, wo.SM) < 1e-9
    eng.close()


def test_engine_configs1_full_population():
    """The FP64 drop-in at M=128, N=32+32, Nchol=640 with all 1024 walkers: run_afqmc's loop for 21
    steps (orthogonalization every 5, combs at steps 0 and 20, Eshift relaxed every step) against
    the oracle on the same Philox fields; weights, overlaps and walkers at 1e-10, the combs
    bit-exact (the same walkers in the same slots).  dt = 0.002: at 0.005 these walkers collapse
    within a few steps, in the oracle as well."""
    s, ham, eng, prop, wo = _engine_pair(synthetic.CFG_MEDIUM, 1024, dt=0.002, seed=7)
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    assert abs(Esh - Esh_o) < REL * abs(Esh_o)
    Esh_o, _ = O.run(ham, wo, prop, 21, Esh_o, ortho_interval=5, pop_interval=20)
    Esh, _ = eng.run(21, Esh, ortho_interval=5, pop_interval=20)
    assert abs(Esh - Esh_o) < REL * abs(Esh_o)
    SM, pr = eng.walkers()
    assert rel(pr["WEIGHT"], wo.weight) < REL
    assert rel(pr["OVLP"], wo.ovlp) < REL
    assert rel(SM, wo.SM) < REL
    # the comb picked the same parents: every slot holds the oracle's walker, not merely a close one
    assert np.max(np.abs(SM - wo.SM)) < 1e-9 * np.max(np.abs(wo.SM))
    eng.close()


def test_engine_configs2_fp64_step_on_a_sample():
    """The FP64 drop-in at M=400, N=100+100, Nchol=2400 on a 16-walker sample: one step and the
    local energy of the propagated walkers against the oracle at 1e-10."""
    s, ham, eng, prop, wo = _engine_pair(synthetic.CFG_LARGE, 16, dt=0.0005, seed=1000)
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    assert abs(Esh - Esh_o) < REL * abs(Esh_o)
    dbg = prop.propagate(wo, Esh_o, 0)
    eng.propagate(Esh, 0)
    assert rel(eng.fetch("X", (16, s.Nc), np.complex128), dbg["X"]) < REL
    SM, pr = eng.walkers()
    assert rel(SM, wo.SM) < REL
    assert rel(pr["WEIGHT"], wo.weight) < REL
    assert rel(pr["OVLP"], wo.ovlp) < REL
    E = eng.energy()
    Eo, _ = O.wfn_energy_noupdate(ham, wo)
    assert rel(E, Eo) < REL
    eng.close()


def test_engine_host_step_matches_device_step():
    s = synthetic.make_system(synthetic.CFG_SMALL)
    e1 = A.AfqmcEngine(s, 8, seed=3)
    e2 = A.AfqmcEngine(s, 8, seed=3)
    Esh = e1.init()
    e2.init()
    props = np.empty((8, 8), np.complex128)
    for step in range(3):  # consecutive host steps: each one's uniforms copied while the last is read
        u = philox.uniforms(3, philox.STREAM_FIELDS, step, 8, s.Nc)
        e1.propagate_host(Esh, step, u, props)
        e2.propagate(Esh, step)
        SM1, p1 = e1.walkers()
        SM2, p2 = e2.walkers()
        assert np.array_equal(SM1, SM2)
        assert np.array_equal(props[0], p2["WEIGHT"])
    e1.close()
    e2.close()


def test_engine_medium_steps():
    """FP64 drop-in at M=128, N=32, Nc=640 on fewer walkers: 4 steps + ortho vs the oracle."""
    s, ham, eng, prop, wo = _engine_pair(synthetic.CFG_MEDIUM, 16)
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    assert abs(Esh - Esh_o) < REL * abs(Esh_o)
    for step in range(4):
        prop.propagate(wo, Esh_o, step)
        eng.propagate(Esh, step)
    eng.orthogonalize()
    prop.orthogonalize(wo)
    SM, pr = eng.walkers()
    assert rel(SM, wo.SM) < REL
    assert rel(pr["WEIGHT"], wo.weight) < REL
    assert rel(pr["OVLP"], wo.ovlp) < REL
    E = eng.energy()
    Eo, _ = O.wfn_energy_noupdate(ham, wo)
    assert rel(E, Eo) < REL
    eng.close()


@pytest.mark.parametrize("symmetric", [True, False])
def test_engine_vhs_packed_and_full_paths(symmetric):
    """Symmetric Cholesky vectors take the packed upper-triangle vHS; any asymmetry the full one.
    Both give the oracle's vHS and step."""
    s = synthetic.make_system(synthetic.CFG_SMALL)
    if not symmetric:
        s.Likn = s.Likn.copy()
        s.Likn[0, 1, :] += 1e-3  # L_n no longer symmetric in (i, k)
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    W = 8
    eng = A.AfqmcEngine(s, W, dt=0.005, seed=2)
    prop = O.Propagator(ham, 0.005, seed=2)
    wo = O.Walkers(s.initial_walkers(W))
    assert eng.info().vhs_packed == (1 if symmetric else 0)
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    dbg = prop.propagate(wo, Esh_o, 0)
    eng.propagate(Esh, 0)
    assert rel(eng.fetch("vHS", (W, s.M, s.M), np.complex128), dbg["vHS"]) < REL
    SM, pr = eng.walkers()
    assert rel(SM, wo.SM) < REL
    assert rel(pr["WEIGHT"], wo.weight) < REL
    eng.close()
