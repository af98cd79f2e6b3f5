"""The reference's input files for the dense closed-shell path: Hamiltonian and NOMSD trial.

    system = load_system("afqmc_H.h5", "afqmc_wfn.h5")     # hcore, Likn, PsiT, E0 as the engine takes them
    eng = AfqmcEngine(system, nwalk=50, dt=0.01)
    wfn = load_nomsd_trial("afqmc_wfn.h5")                 # or the pieces: PsiT (nel, nmo) complex
    ham = load_dense_hamiltonian("afqmc_H.h5", nup=wfn["nup"])

Layouts (read with safire_b200.h5read):

  Hamiltonian/hcore                [nspin][npol][NMO][npol][NMO] real (or a trailing 2 for complex)
  Hamiltonian/DenseFactorized/L    [nspin][1][NMO][1][NMO][nchol] real
  Hamiltonian attributes           nuclear_energy, frozen_core_energy, madelung_constant
                                   (read_energy_offset, hdf5_helpers.hpp:84-106)
  Wavefunction/NOMSD               attribute spin_type; ci_coeffs; PsiT_<i> as CSR, either
                                   shape / row_pointers / column_indices / values, or the legacy
                                   dims / pointers_begin_ / pointers_end_ / jdata_ / data_
                                   (csr_utils.hpp:345-420)

The reference's readers: RealDenseHamiltonian::getHamiltonianOperations
(RealDenseHamiltonian.cpp:77-134) and read_wavefunction_info / HDF2CSR (readWfn.cpp:50-131,
csr_utils.hpp:372-420).  Only what the dense real-Cholesky path uses is accepted (CLOSED, COLLINEAR and
NONCOLLINEAR walkers over a spin-independent Hamiltonian; NOMSD trials of one or several
determinants); anything else raises InputError with the reason, as utils::check aborts there.
"""
import numpy as np

from .h5read import H5File


class InputError(ValueError):
    pass


def _check(cond, msg):
    if not cond:
        raise InputError(msg)


def _complex_last(a, rank):
    """A dataset of the given rank, or the same with a trailing 2 for interleaved complex values."""
    a = np.asarray(a)
    if a.ndim == rank + 1 and a.shape[-1] == 2 and not np.iscomplexobj(a):
        return a[..., 0] + 1j * a[..., 1]
    return a


def energy_offset(f, nup, ndn=0, closed=True):
    """read_energy_offset (hdf5_helpers.hpp:84-106): nuclear + frozen core - madelung * nelec, nelec
    2 nup for CLOSED walkers, nup + ndn otherwise (NONCOLLINEAR: nup is every electron, ndn 0)."""
    at = f.attrs("Hamiltonian")
    nuc = float(at.get("nuclear_energy", 0.0))
    fzc = float(at.get("frozen_core_energy", 0.0))
    mad = 0.0
    if "madelung_constant" in at:
        nelec = 2 * nup if closed else nup + ndn
        mad = -1.0 * nelec * float(at["madelung_constant"])
    return nuc + fzc + mad


def load_dense_hamiltonian(path, nup, ndn=None):
    """hcore (nmo, nmo) real, Likn (nmo, nmo, nchol) real and E0 of a dense Cholesky Hamiltonian;
    ndn None: CLOSED walkers with nup electrons per spin, else nup up and ndn down electrons."""
    f = H5File(path)
    _check("Hamiltonian" in f, f"{path}: no Hamiltonian group")
    _check("Hamiltonian/DenseFactorized/L" in f, f"{path}: not a dense factorized Hamiltonian "
           "(Hamiltonian/DenseFactorized/L missing)")
    h = _complex_last(f["Hamiltonian/hcore"], 5)
    _check(h.ndim == 5, f"hcore has rank {h.ndim}, expected [nspin][npol][NMO][npol][NMO]")
    nspin, npol, nmo = h.shape[0], h.shape[1], h.shape[2]
    _check(h.shape == (nspin, npol, nmo, npol, nmo), f"hcore has shape {h.shape}")
    _check(nspin == 1 and npol == 1, f"hcore with nspin={nspin}, npol={npol}: CLOSED walkers take nspin = npol = 1")
    hc = h[0, 0, :, 0, :]
    if np.iscomplexobj(hc):
        _check(not np.any(hc.imag), "complex hcore: the dense real-Cholesky path takes a real one-body term")
        hc = hc.real
    L = np.asarray(f["Hamiltonian/DenseFactorized/L"])
    _check(L.ndim == 6, f"DenseFactorized/L has rank {L.ndim}")
    _check(L.shape[1] == 1 and L.shape[3] == 1, f"spinor Cholesky vectors (npol: {L.shape[1]}) are not supported")
    _check(L.shape[0] == 1 and L.shape[2] == nmo and L.shape[4] == nmo,
           f"DenseFactorized/L has shape {L.shape}, expected (1, 1, {nmo}, 1, {nmo}, nchol)")
    _check(not np.iscomplexobj(L), "DenseFactorized/L must be real")
    Likn = np.ascontiguousarray(L[0, 0, :, 0, :, :], dtype=np.float64)
    return dict(hcore=np.ascontiguousarray(hc, dtype=np.float64), Likn=Likn,
                E0=energy_offset(f, nup, ndn or 0, closed=ndn is None), nmo=nmo, nchol=Likn.shape[2])


def read_csr(f, group):
    """HDF2CSR (csr_utils.hpp:372-420) to a dense complex matrix."""
    legacy = f"{group}/shape" not in f
    if legacy:
        dims = np.asarray(f[f"{group}/dims"]).astype(np.int64)
        _check(dims.size == 3, f"sparse matrix 'dims' has length {dims.size}, expected 3")
        nrows, ncols, nnz = (int(x) for x in dims)
        ptrb = np.asarray(f[f"{group}/pointers_begin_"]).astype(np.int64)
        ptre = np.asarray(f[f"{group}/pointers_end_"]).astype(np.int64)
        vals = _complex_last(f[f"{group}/data_"], 1)
        cols = np.asarray(f[f"{group}/jdata_"]).astype(np.int64)
    else:
        shape = np.asarray(f[f"{group}/shape"]).astype(np.int64)
        _check(shape.size == 2, f"sparse matrix 'shape' has length {shape.size}, expected 2")
        nrows, ncols = (int(x) for x in shape)
        rp = np.asarray(f[f"{group}/row_pointers"]).astype(np.int64)
        _check(rp.size == nrows + 1, f"row_pointers has {rp.size} entries, expected {nrows + 1}")
        _check(rp[0] == 0, f"row_pointers starts at {rp[0]}, expected 0")
        nnz = int(rp[-1])
        ptrb, ptre = rp[:-1], rp[1:]
        vals = _complex_last(f[f"{group}/values"], 1)
        cols = np.asarray(f[f"{group}/column_indices"]).astype(np.int64)
    _check(ptrb.size == nrows and ptre.size == nrows, "row pointer arrays do not match the row count")
    _check(vals.size >= nnz and cols.size >= nnz, f"{group}: fewer stored values than nnz = {nnz}")
    A = np.zeros((nrows, ncols), np.complex128)
    for r in range(nrows):
        for i in range(int(ptrb[r]), int(ptre[r])):
            c = int(cols[i])
            _check(0 <= c < ncols, f"{group}: column index {c} outside [0, {ncols})")
            A[r, c] += vals[i]  # emplace_back of a repeated (row, col) adds
    return A


def _spinors(up, dn):
    """combine_csr (csr_utils.hpp:70-110): the up rows over the down rows, the latter shifted by nmo."""
    M = up.shape[1]
    sp = np.zeros((up.shape[0] + dn.shape[0], 2 * M), np.complex128)
    sp[:up.shape[0], :M] = up
    sp[up.shape[0]:, M:] = dn
    return sp


def load_nomsd_determinants(path, walker_type="CLOSED"):
    """Every determinant of a NOMSD trial for the given walker type, upgraded as
    read_nomsd_wavefunction does (readWfn.h:90-153): a list of dicts (PsiT; COLLINEAR also PsiT_up,
    PsiT_dn) and the coefficients ci.  A closed file gives COLLINEAR walkers the same orbitals for
    both spins and NONCOLLINEAR walkers the spinor matrix of both; a collinear file gives
    NONCOLLINEAR walkers its up and down rows as spinors."""
    walker_type = walker_type.upper()
    _check(walker_type in ("CLOSED", "COLLINEAR", "NONCOLLINEAR"), f"unknown walker type {walker_type}")
    f = H5File(path)
    _check("Wavefunction/NOMSD" in f, f"{path}: no Wavefunction/NOMSD group")
    spin = f.attrs("Wavefunction/NOMSD").get("spin_type")
    spin = str(spin).lower() if spin is not None else walker_type.lower()
    order = ("closed", "collinear", "noncollinear")  # walkerTypeIsConvertible: upgrades only
    _check(spin in order and order.index(spin) <= order.index(walker_type.lower()),
           f"wavefunction spin_type is '{spin}': {walker_type} walkers cannot take it")
    ci = np.atleast_1d(_complex_last(f["Wavefunction/NOMSD/ci_coeffs"], 1))
    per = 2 if spin == "collinear" else 1
    dets = []
    for d in range(ci.size):
        g = f"Wavefunction/NOMSD/PsiT_{per * d}"
        _check(g in f, f"{g} missing")
        P = read_csr(f, g)
        dn = read_csr(f, f"Wavefunction/NOMSD/PsiT_{per * d + 1}") if spin == "collinear" else None
        if walker_type == "NONCOLLINEAR":
            if spin == "noncollinear":
                _check(P.shape[1] % 2 == 0, f"noncollinear {g} has {P.shape[1]} columns, not 2 nmo")
                dets.append(dict(PsiT=P, nup=P.shape[0], nmo=P.shape[1] // 2))
            else:
                sp = _spinors(P, dn if dn is not None else P)
                dets.append(dict(PsiT=sp, nup=sp.shape[0], nmo=P.shape[1]))
        elif walker_type == "COLLINEAR":
            dn = P if dn is None else dn
            _check(dn.shape[1] == P.shape[1], f"{g}: up and down orbitals differ in nmo")
            dets.append(dict(PsiT=P, PsiT_up=P, PsiT_dn=dn, nup=P.shape[0], ndn=dn.shape[0], nmo=P.shape[1]))
        else:
            dets.append(dict(PsiT=P, nup=P.shape[0], nmo=P.shape[1]))
    return dets, ci.astype(np.complex128), spin


def load_nomsd_trial(path, walker_type="CLOSED"):
    """A single-determinant NOMSD trial: for CLOSED walkers PsiT (nel, nmo) complex; for COLLINEAR
    walkers also PsiT_up (nup, nmo) and PsiT_dn (ndn, nmo), ndn possibly 0; for NONCOLLINEAR walkers
    PsiT (nel, 2 nmo) spinors.  Trials are upgraded as load_nomsd_determinants says."""
    dets, ci, spin = load_nomsd_determinants(path, walker_type)
    _check(ci.size == 1, f"{ci.size} determinants: the path takes a single-determinant trial")
    out = dict(dets[0])
    out.update(ci=complex(ci[0]), spin_type=spin)
    return out


def load_system(hamiltonian_path, wavefunction_path, walker_type="CLOSED"):
    """The engine's System (hcore, Likn, PsiT, E0 and sizes) from a Hamiltonian and a NOMSD trial file,
    for CLOSED, COLLINEAR and NONCOLLINEAR walkers and single- or multi-determinant trials, as
    getHamiltonianOperations and read_nomsd_wavefunction take them (RealDenseHamiltonian.cpp:77-134,
    readWfn.h:90-153): COLLINEAR PsiT stacks the up rows over the down rows and nel_dn counts the
    latter; NONCOLLINEAR PsiT holds the (N, 2 nmo) spinor orbitals (npol 2); a trial of several
    determinants gives PsiT (ndet, rows, cols) and the coefficients ci.  E0 counts the electrons as
    read_energy_offset does for the walker type."""
    from .synthetic import System, SystemSpec
    wt = walker_type.upper()
    dets, ci, _ = load_nomsd_determinants(wavefunction_path, wt)
    d0 = dets[0]
    kw = {}
    if wt == "COLLINEAR":
        ham = load_dense_hamiltonian(hamiltonian_path, d0["nup"], d0["ndn"])
        for d in dets:
            _check((d["nup"], d["ndn"]) == (d0["nup"], d0["ndn"]),
                   f"determinants with {d['nup']} + {d['ndn']} and {d0['nup']} + {d0['ndn']} electrons")
        mats = [np.concatenate([d["PsiT_up"], d["PsiT_dn"]]) for d in dets]
        kw["nel_dn"] = d0["ndn"]
    elif wt == "NONCOLLINEAR":
        ham = load_dense_hamiltonian(hamiltonian_path, d0["nup"], 0)
        mats = [d["PsiT"] for d in dets]
        kw["npol"] = 2
    else:
        ham = load_dense_hamiltonian(hamiltonian_path, d0["nup"])
        mats = [d["PsiT"] for d in dets]
    _check(d0["nmo"] == ham["nmo"], f"trial has {d0['nmo']} orbitals, Hamiltonian {ham['nmo']}")
    for m in mats:
        _check(m.shape == mats[0].shape, f"determinants of shapes {m.shape} and {mats[0].shape}")
    N = mats[0].shape[0]
    if len(mats) > 1:
        PsiT = np.stack(mats)
        kw["ci"] = ci
    else:
        PsiT = mats[0]
    spec = SystemSpec(M=ham["nmo"], N=N, Nc=ham["nchol"], decay=0.0)
    return System(spec, ham["hcore"], ham["Likn"], PsiT, ham["E0"], **kw)
