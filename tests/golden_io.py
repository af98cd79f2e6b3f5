"""Helpers that load the committed golden fixtures."""
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cplx(a):
    a = np.asarray(a, dtype=np.float64)
    return a[..., 0] + 1j * a[..., 1]


def sdet_kats():
    with open(os.path.join(HERE, "sdet_kats.json")) as f:
        k = json.load(f)
    out = {}
    for key, v in k.items():
        if isinstance(v, list):
            out[key] = cplx(v)
        else:
            out[key] = v
    return out


SNAPSHOT_OBSERVABLES = ("Energy", "OnebodyEnergy", "ExchangeEnergy", "CoulombEnergy", "Overlap", "ProjectionTime",
                        "EffectiveNumWalkers", "Phase", "TotalWeight")


def snapshot(name):
    """A seeded snapshot case (make_bh_snapshot.py): inputs, settings and recorded (mean, error).
    The BH collinear case shares the BH Hamiltonian tensors of the closed case's file."""
    z = np.load(os.path.join(HERE, f"{name}_snapshot.npz"))
    rec = {k: (z[f"mean_{k}"][()], z[f"error_{k}"][()]) for k in SNAPSHOT_OBSERVABLES}
    rdm = ["MixedEstimator/OneRDM", "MixedEstimator/DiagonalTwoRDM"]
    bp_steps = [int(k) for k in z["bp_steps"]] if "bp_steps" in z else []
    rdm += [f"BackPropEstimator/Steps={k}/{o}" for k in bp_steps for o in ("OneRDM", "DiagonalTwoRDM")]
    for k in rdm:
        key = k.replace("/", "_").replace("=", "")
        if f"mean_{key}" in z:
            rec[k] = (z[f"mean_{key}"], z[f"error_{key}"])
    out = dict(settings=json.loads(str(z["settings"])), recorded=rec,
               mixed_interval=int(z["mixed_interval"]) if "mixed_interval" in z else None,
               bp_steps=bp_steps or None,
               bp_ortho_interval=int(z["bp_ortho_interval"]) if "bp_ortho_interval" in z else None)
    if "ci_dets" in z:  # multi-determinant trial: per-determinant orbitals and coefficients
        out.update(ci_dets=z["ci_dets"], PsiT_dets=z["PsiT_dets"])
        if "PsiT_up_dets" in z:
            out.update(PsiT_up_dets=z["PsiT_up_dets"], PsiT_dn_dets=z["PsiT_dn_dets"])
    else:
        out.update(PsiT=z["PsiT"], ci=complex(z["ci"]))
        if "PsiT_up" in z:
            out.update(PsiT_up=z["PsiT_up"], PsiT_dn=z["PsiT_dn"])
    h = z if "hcore" in z else np.load(os.path.join(HERE, "bh_rhf_closed_snapshot.npz"))
    out.update(hcore=h["hcore"], Likn=h["Likn"], E0=float(z["E0"]) if "E0" in z else float(h["E0"]))
    return out


def bh_snapshot():
    """The BH CLOSED case."""
    return snapshot("bh_rhf_closed")


def snapshot_match(series, recorded, rebinned_average, tol=1e-9):
    """The rebin size at which the series reproduces the recorded mean and error the way the
    reference's snapshot comparison does (np.allclose, rtol = atol = 1e-9), or None.  The recorded
    numbers came from safiretools' own choice of rebin size; every size with at least two bins is
    tried."""
    m_ref, e_ref = recorded
    for B in range(1, len(series) // 2 + 1):
        m, e = rebinned_average(series, B)
        if np.allclose(m, m_ref, rtol=tol, atol=tol) and np.allclose(e, e_ref, rtol=tol, atol=tol):
            return B
    return None


def bh_statistical(name="bh_rhf_closed"):
    """A statistical reference (make_bh_snapshot.py): settings and recorded mean / error."""
    with open(os.path.join(HERE, f"{name}_statistical.json")) as f:
        s = json.load(f)
    s["recorded"] = {k: (complex(*v["mean"]), complex(*v["error"])) for k, v in s["recorded"].items()}
    return s


def statistically_equal(a, a_err, b, b_err, significance=0.001, components=1):
    """The reference's statistical comparison (run_functional.py:384-412): |a - b| within
    z * sqrt(|a_err|^2 + |b_err|^2), z the two-sided normal quantile at the Bonferroni-adjusted
    significance, or within 1e-9 * (1 + |b|)."""
    from scipy.stats import norm
    z = norm.ppf(1 - significance / (2 * components))
    tol = max(z * float(np.hypot(abs(a_err), abs(b_err))), 1e-9 * (1 + abs(b)))
    return abs(a - b) <= tol, abs(a - b), tol


def oracle_hamiltonian(snap):
    """The oracle's Hamiltonian for a snapshot case: the walker type's class, or their
    multi-determinant combination."""
    from oracle import afqmc_oracle as O
    wt = snap["settings"]["walker_type"]

    def one(PsiT=None, up=None, dn=None, ci=1.0):
        if wt == "NONCOLLINEAR":
            return O.NoncollinearHamiltonian(snap["hcore"], snap["Likn"], PsiT, snap["E0"], ci)
        if wt == "COLLINEAR":
            return O.CollinearHamiltonian(snap["hcore"], snap["Likn"], up, dn, snap["E0"], ci)
        return O.Hamiltonian(snap["hcore"], snap["Likn"], PsiT, snap["E0"])

    if "ci_dets" in snap:
        n = len(snap["ci_dets"])
        if wt == "COLLINEAR":
            dets = [one(up=snap["PsiT_up_dets"][d], dn=snap["PsiT_dn_dets"][d]) for d in range(n)]
        else:
            dets = [one(PsiT=snap["PsiT_dets"][d]) for d in range(n)]
        return O.MultiDetHamiltonian(dets, snap["ci_dets"])
    return one(PsiT=snap["PsiT"], up=snap.get("PsiT_up"), dn=snap.get("PsiT_dn"), ci=snap["ci"])


def engine_system(snap):
    """The engine's System for a snapshot case: COLLINEAR stacks the up rows over the down rows,
    NONCOLLINEAR takes the (N, 2M) spinor trial, a multi-determinant trial stacks its determinants."""
    from safire_b200 import synthetic
    wt = snap["settings"]["walker_type"]
    M, Nc = snap["hcore"].shape[0], snap["Likn"].shape[2]
    kw = {}
    if "ci_dets" in snap:
        if wt == "COLLINEAR":
            PsiT = np.concatenate([snap["PsiT_up_dets"], snap["PsiT_dn_dets"]], axis=1)
            kw["nel_dn"] = snap["PsiT_dn_dets"].shape[1]
        else:
            PsiT = snap["PsiT_dets"]
        kw["ci"] = snap["ci_dets"]
        N = PsiT.shape[1]
    elif wt == "COLLINEAR":
        PsiT = np.concatenate([snap["PsiT_up"], snap["PsiT_dn"]])
        kw["nel_dn"] = snap["PsiT_dn"].shape[0]
        N = PsiT.shape[0]
    else:
        PsiT = snap["PsiT"]
        N = PsiT.shape[0]
    if wt == "NONCOLLINEAR":
        kw["npol"] = 2
    spec = synthetic.SystemSpec(M=M, N=N, Nc=Nc, decay=0.0)
    return synthetic.System(spec, snap["hcore"], snap["Likn"], PsiT, snap["E0"], **kw)
