"""The HDF5 reader and the input loaders on files written here (no reference tree needed).

tests/h5write.py writes the layouts the reference's readers take (RealDenseHamiltonian.cpp:77-134,
hdf5_helpers.hpp:84-106; Wavefunction/NOMSD as readWfn.cpp:50-131 and csr_utils.hpp:345-420 read
it); these tests check that the loaders turn them into the engine's arrays for every walker type,
upgrade trials as read_nomsd_wavefunction does (readWfn.h:90-153), count electrons in the energy
offset per walker type, and refuse what the dense real-Cholesky path does not take.  The loaders
are also checked against the reference's own files in tests/test_snapshot.py where that tree is
present."""
import numpy as np
import pytest

from safire_b200.h5read import H5File
from safire_b200.inputs import (InputError, load_dense_hamiltonian, load_nomsd_determinants, load_nomsd_trial,
                                load_system)
from tests.h5write import write

M, NC = 6, 10
NUC, FZC, MAD = 1.5, -0.25, 0.125


def _rng(seed=3):
    return np.random.default_rng(seed)


def _hamiltonian(path, hcore=None, L=None, attrs=None):
    r = _rng()
    if hcore is None:
        h = r.normal(size=(M, M))
        hcore = (h + h.T)[None, None, :, None, :]
    if L is None:
        L = r.normal(size=(M, M, NC))
        L = (L + L.transpose(1, 0, 2))[None, None, :, None, :, :]
    write(path, {"Hamiltonian/hcore": hcore, "Hamiltonian/DenseFactorized/L": L},
          attrs={"Hamiltonian": attrs if attrs is not None else
                 {"nuclear_energy": NUC, "frozen_core_energy": FZC, "madelung_constant": MAD}})
    return hcore, L


def _cplx2(z):
    return np.stack([z.real, z.imag], axis=-1)


def _csr(P, legacy=False, drop=True):
    """PsiT as the reference stores it: CSR of the nonzeros (explicit zeros dropped)."""
    cols, vals = [], []
    ptr = [0]
    for i in range(P.shape[0]):
        for j in range(P.shape[1]):
            if P[i, j] != 0 or not drop:
                cols.append(j)
                vals.append(P[i, j])
        ptr.append(len(cols))
    vals = _cplx2(np.asarray(vals, np.complex128).reshape(-1))
    if legacy:
        return {"dims": np.array([P.shape[0], P.shape[1], len(cols)]), "pointers_begin_": np.array(ptr[:-1]),
                "pointers_end_": np.array(ptr[1:]), "jdata_": np.array(cols), "data_": vals}
    return {"shape": np.array(P.shape), "row_pointers": np.array(ptr), "column_indices": np.array(cols), "values": vals}


def _trial(r, n, m):
    P = r.normal(size=(n, m)) + 1j * r.normal(size=(n, m))
    P[r.random(P.shape) < 0.3] = 0.0  # a sparse trial, as CSR files hold them
    return P


def _wavefunction(path, dets, ci, spin, legacy=False):
    """dets: list of PsiT (one per determinant; COLLINEAR: (up, down) pairs)."""
    data = {"Wavefunction/NOMSD/ci_coeffs": _cplx2(np.asarray(ci, np.complex128))}
    k = 0
    for d in dets:
        for P in (d if isinstance(d, tuple) else (d,)):
            for name, v in _csr(P, legacy).items():
                data[f"Wavefunction/NOMSD/PsiT_{k}/{name}"] = v
            k += 1
    write(path, data, attrs={"Wavefunction/NOMSD": {"spin_type": spin}})


def test_h5read_reads_the_written_layout(tmp_path):
    p = str(tmp_path / "x.h5")
    a = np.arange(24, dtype=np.float64).reshape(2, 3, 4) / 7
    write(p, {"g/a": a, "g/h/i": np.array([3, -1, 2**40]), "g/h/e": np.zeros((0,)), "top": np.array(2.5)},
          attrs={"g": {"x": 1.25, "name": "collinear"}, "g/h/i": {"n": 7}})
    f = H5File(p)
    assert f.keys() == ["g", "top"] and f.keys("g") == ["a", "h"] and f.keys("g/h") == ["e", "i"]
    assert f.is_group("g/h") and not f.is_group("g/a")
    assert np.array_equal(f["g/a"], a) and f.shape("g/a") == (2, 3, 4)
    assert np.array_equal(f["g/h/i"], [3, -1, 2**40]) and f["g/h/e"].shape == (0,)
    assert f["top"] == 2.5
    assert f.attrs("g") == {"x": 1.25, "name": "collinear"} and f.attrs("g/h/i") == {"n": 7}
    assert "g/h" in f and "g/z" not in f


@pytest.mark.parametrize("legacy", [False, True])
def test_closed_trial_for_every_walker_type(tmp_path, legacy):
    r = _rng(5)
    hcore, L = _hamiltonian(str(tmp_path / "H.h5"))
    P = _trial(r, 3, M)
    _wavefunction(str(tmp_path / "W.h5"), [P], [1.0], "closed", legacy)
    H, Wf = str(tmp_path / "H.h5"), str(tmp_path / "W.h5")
    s = load_system(H, Wf, "CLOSED")
    assert (s.M, s.N, s.Nc, s.nel_dn, s.npol, s.ci) == (M, 3, NC, -1, 1, None)
    assert np.array_equal(s.PsiT, P) and np.array_equal(s.hcore, hcore[0, 0, :, 0, :])
    assert np.array_equal(s.Likn, L[0, 0, :, 0, :, :])
    assert s.E0 == NUC + FZC - 2 * 3 * MAD  # read_energy_offset: 2 nup electrons for CLOSED walkers
    c = load_system(H, Wf, "COLLINEAR")  # upgraded: the same orbitals for both spins
    assert (c.N, c.nel_dn) == (6, 3) and np.array_equal(c.PsiT, np.concatenate([P, P]))
    assert c.E0 == NUC + FZC - 6 * MAD
    n = load_system(H, Wf, "NONCOLLINEAR")  # upgraded: spinors [[P, 0], [0, P]]
    assert (n.N, n.npol) == (6, 2) and n.PsiT.shape == (6, 2 * M)
    assert np.array_equal(n.PsiT[:3, :M], P) and np.array_equal(n.PsiT[3:, M:], P)
    assert not n.PsiT[:3, M:].any() and not n.PsiT[3:, :M].any()
    assert n.E0 == NUC + FZC - 6 * MAD


def test_collinear_and_noncollinear_trials(tmp_path):
    r = _rng(7)
    _hamiltonian(str(tmp_path / "H.h5"))
    H = str(tmp_path / "H.h5")
    up, dn = _trial(r, 3, M), _trial(r, 2, M)
    _wavefunction(str(tmp_path / "U.h5"), [(up, dn)], [1.0], "collinear")
    c = load_system(H, str(tmp_path / "U.h5"), "COLLINEAR")
    assert (c.N, c.nel_dn) == (5, 2) and np.array_equal(c.PsiT, np.concatenate([up, dn]))
    assert c.E0 == NUC + FZC - 5 * MAD
    n = load_system(H, str(tmp_path / "U.h5"), "NONCOLLINEAR")
    assert np.array_equal(n.PsiT[:3, :M], up) and np.array_equal(n.PsiT[3:, M:], dn)
    with pytest.raises(InputError):  # a collinear trial does not fit CLOSED walkers
        load_system(H, str(tmp_path / "U.h5"), "CLOSED")
    G = _trial(r, 5, 2 * M)
    _wavefunction(str(tmp_path / "G.h5"), [G], [1.0], "noncollinear")
    g = load_system(H, str(tmp_path / "G.h5"), "NONCOLLINEAR")
    assert (g.N, g.npol) == (5, 2) and np.array_equal(g.PsiT, G) and g.E0 == NUC + FZC - 5 * MAD
    for wt in ("CLOSED", "COLLINEAR"):
        with pytest.raises(InputError):
            load_system(H, str(tmp_path / "G.h5"), wt)


def test_multi_determinant_trials(tmp_path):
    r = _rng(11)
    _hamiltonian(str(tmp_path / "H.h5"))
    H = str(tmp_path / "H.h5")
    dets = [_trial(r, 3, M) for _ in range(4)]
    ci = r.normal(size=4) + 1j * r.normal(size=4)
    _wavefunction(str(tmp_path / "D.h5"), dets, ci, "closed")
    s = load_system(H, str(tmp_path / "D.h5"), "CLOSED")
    assert s.PsiT.shape == (4, 3, M) and np.array_equal(s.PsiT, np.stack(dets)) and np.array_equal(s.ci, ci)
    n = load_system(H, str(tmp_path / "D.h5"), "NONCOLLINEAR")
    assert n.PsiT.shape == (4, 6, 2 * M) and np.array_equal(n.ci, ci)
    for d in range(4):
        assert np.array_equal(n.PsiT[d, :3, :M], dets[d]) and np.array_equal(n.PsiT[d, 3:, M:], dets[d])
    pairs = [(_trial(r, 3, M), _trial(r, 2, M)) for _ in range(3)]
    _wavefunction(str(tmp_path / "E.h5"), pairs, ci[:3], "collinear")
    c = load_system(H, str(tmp_path / "E.h5"), "COLLINEAR")
    assert c.PsiT.shape == (3, 5, M) and c.nel_dn == 2
    for d, (u, v) in enumerate(pairs):
        assert np.array_equal(c.PsiT[d], np.concatenate([u, v]))
    with pytest.raises(InputError):  # the single-determinant reader refuses several
        load_nomsd_trial(str(tmp_path / "D.h5"))
    dets_, ci_, spin = load_nomsd_determinants(str(tmp_path / "D.h5"), "COLLINEAR")
    assert spin == "closed" and len(dets_) == 4 and np.array_equal(ci_, ci)
    assert all(np.array_equal(d["PsiT_up"], d["PsiT_dn"]) for d in dets_)


def test_csr_repeated_entries_add_and_bad_indices_are_refused(tmp_path):
    _hamiltonian(str(tmp_path / "H.h5"))
    base = {"Wavefunction/NOMSD/ci_coeffs": _cplx2(np.array([1.0 + 0j]))}
    attrs = {"Wavefunction/NOMSD": {"spin_type": "closed"}}
    vals = _cplx2(np.array([1.0, 2.0 + 1j, 0.5]))
    g = "Wavefunction/NOMSD/PsiT_0"
    # row 0 holds (0, 1) twice: emplace_back of a repeated entry adds
    write(str(tmp_path / "R.h5"), {**base, f"{g}/shape": np.array([2, M]), f"{g}/row_pointers": np.array([0, 2, 3]),
                                   f"{g}/column_indices": np.array([1, 1, 4]), f"{g}/values": vals}, attrs)
    P = load_nomsd_trial(str(tmp_path / "R.h5"))["PsiT"]
    want = np.zeros((2, M), np.complex128)
    want[0, 1], want[1, 4] = 3.0 + 1j, 0.5
    assert np.array_equal(P, want)
    for rp, cols, why in (([1, 2, 3], [1, 1, 4], "row_pointers"), ([0, 2, 3], [1, M, 4], "column index"),
                          ([0, 2], [1, 1, 4], "entries")):
        write(str(tmp_path / "B.h5"), {**base, f"{g}/shape": np.array([2, M]), f"{g}/row_pointers": np.array(rp),
                                       f"{g}/column_indices": np.array(cols), f"{g}/values": vals}, attrs)
        with pytest.raises(InputError, match=why):
            load_nomsd_trial(str(tmp_path / "B.h5"))


def test_what_the_dense_real_path_does_not_take_is_refused(tmp_path):
    r = _rng(13)
    H = str(tmp_path / "H.h5")
    hc = r.normal(size=(1, 2, M, 2, M))  # spinor one-body term (npol = 2)
    _hamiltonian(H, hcore=hc)
    with pytest.raises(InputError, match="npol"):
        load_dense_hamiltonian(H, 3)
    _hamiltonian(H, L=r.normal(size=(1, 1, M, 1, M, NC, 2)))  # complex Cholesky vectors (re, im last)
    with pytest.raises(InputError, match="rank 7"):
        load_dense_hamiltonian(H, 3)
    hcx = np.zeros((1, 1, M, 1, M, 2))
    hcx[0, 0, :, 0, :, 0] = np.eye(M)
    hcx[0, 0, 0, 0, 1, 1] = 0.5  # a complex one-body term
    _hamiltonian(H, hcore=hcx)
    with pytest.raises(InputError, match="complex hcore"):
        load_dense_hamiltonian(H, 3)
    write(H, {"Hamiltonian/hcore": np.eye(M)[None, None, :, None, :]}, attrs={"Hamiltonian": {"nuclear_energy": 0.0}})
    with pytest.raises(InputError, match="DenseFactorized"):  # another factorization
        load_dense_hamiltonian(H, 3)
    _hamiltonian(H, attrs={"nuclear_energy": NUC})  # no frozen core or Madelung term
    assert load_dense_hamiltonian(H, 3)["E0"] == NUC
    _wavefunction(str(tmp_path / "W.h5"), [_trial(r, 3, M + 1)], [1.0], "closed")
    with pytest.raises(InputError, match="orbitals"):  # trial and Hamiltonian disagree on nmo
        load_system(H, str(tmp_path / "W.h5"))
