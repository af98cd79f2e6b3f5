"""Extract the dense-Cholesky NOMSD cases of the reference's functional tests: the seeded snapshots
of BH with CLOSED walkers (bh_rhf_closed_snapshot.npz), BH with a UHF trial and COLLINEAR walkers
(bh_uhf_collinear_snapshot.npz), BH with the RHF trial and COLLINEAR walkers
(bh_rhf_collinear_snapshot.npz), BH with NONCOLLINEAR walkers and the RHF, UHF and GHF trials
(bh_{rhf,uhf,ghf}_noncollinear_snapshot.npz), BH with multi-determinant CASCI trials
(bh_rcasci_*_snapshot.npz), Li with a polarized ROHF trial and COLLINEAR walkers
(li_rohf_collinear_snapshot.npz), and the statistical reference of the first (bh_rhf_closed_statistical.json).

    python tests/golden/make_bh_snapshot.py [SAFIRE source tree]

The BH closed case (tests/functional/run_functional.py:195-245 with --snapshot; functional_cases.py:101-134):
Hamiltonian afqmc_inputs/BH/afqmc_H_rhf_closed.h5 (dense Cholesky), trial afqmc_inputs/BH/afqmc_rhf_nomsd.h5
(RHF, NOMSD, one determinant), CLOSED walkers, seed 42, 50 walkers, timestep 0.01, 20 steps, population
control and measurement every step, orthogonalization every 10 steps, no equilibration, one rank.  The
recorded results are snapshot_references/BH/dense_rhf_basis_closed/rhf_nomsd/closed/results.h5: for each
observable the mean and error of its rebinned series (safiretools Results.average).

The collinear cases have the same settings (functional_cases.py:101-143).  Stored per case: the
Hamiltonian and trial as the engine takes them (read by safire_b200.inputs), the run settings, and the
recorded mean / error of every observable of the energy estimator.  The
back-propagated and mixed RDM estimators the case also recorded are outside the path and not stored.

The statistical reference (statistical_references/BH/dense_rhf_basis_closed/rhf_nomsd/closed/results.h5)
is the same case run long: its settings (walkers per rank x ranks, steps, equilibration, intervals) and
the mean / error of the energy observables after equilibration.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from safire_b200.h5read import H5File  # noqa: E402
from safire_b200.inputs import load_dense_hamiltonian, load_nomsd_determinants, load_nomsd_trial  # noqa: E402

OBSERVABLES = ("Energy", "OnebodyEnergy", "ExchangeEnergy", "CoulombEnergy", "Overlap", "ProjectionTime",
               "EffectiveNumWalkers", "Phase", "TotalWeight")
# the RDM estimators of the back-propagation cases: their mixed and back-propagated observables
RDM_OBSERVABLES = ("MixedEstimator/OneRDM", "MixedEstimator/DiagonalTwoRDM")


def rdm_records(res, ex, out):
    """The mixed estimator's recorded RDMs and its measure interval, where the case has them."""
    est = ex.get("estimators")
    if not est or "mixed" not in est:
        return
    out["mixed_interval"] = np.int64(est["mixed"]["measure_interval"])
    obs = list(RDM_OBSERVABLES)
    bp = est.get("backprop")
    if bp:
        steps = [int(k) for k in bp["propagation_steps"]]
        out["bp_steps"] = np.asarray(steps, np.int64)
        out["bp_ortho_interval"] = np.int64(bp.get("walker_ortho_interval", ex["walker_ortho_interval"]))
        out["bp_path_restoration"] = np.int64(bool(bp.get("path_restoration", True)))
        obs += [f"BackPropEstimator/Steps={k}/{o}" for k in steps for o in ("OneRDM", "DiagonalTwoRDM")]
    for k in obs:
        key = k.replace("/", "_").replace("=", "")
        out[f"mean_{key}"] = np.asarray(res[f"measurements/Stage0/{k}/mean"])
        out[f"error_{key}"] = np.asarray(res[f"measurements/Stage0/{k}/error"])


def snapshot_case(fn, system, ham_file, wfn_file, case, walker_type, out_name, with_hamiltonian=True):
    """One seeded snapshot case: inputs as the engine takes them, settings, recorded mean / error."""
    wfn = load_nomsd_trial(os.path.join(fn, "afqmc_inputs", system, wfn_file), walker_type)
    ndn = None if walker_type == "CLOSED" else (wfn.get("ndn", 0))
    ham = load_dense_hamiltonian(os.path.join(fn, "afqmc_inputs", system, ham_file), wfn["nup"], ndn)
    res = H5File(os.path.join(fn, "snapshot_references", system, *case.split("/"), "results.h5"))
    inp = json.loads(res["input_file"])
    ex = inp["execute"]
    settings = dict(seed=inp["seed"], nwalk=ex["num_walkers"], dt=ex["timestep"], steps=ex["steps"],
                    ortho_interval=ex["walker_ortho_interval"], pop_interval=ex["population_control_interval"],
                    measure_interval=ex["measure_interval"], equilibration_steps=ex["equilibration_steps"],
                    num_ranks=int(res["num_ranks"]), walker_type=ex["walker_set"]["walker_type"])
    assert settings["walker_type"] == walker_type
    out = dict(PsiT=wfn["PsiT"], E0=np.float64(ham["E0"]), ci=np.complex128(wfn["ci"]), settings=json.dumps(settings))
    if walker_type == "COLLINEAR":
        out.update(PsiT_up=wfn["PsiT_up"], PsiT_dn=wfn["PsiT_dn"])
    if with_hamiltonian:
        out.update(hcore=ham["hcore"], Likn=ham["Likn"])
    for k in OBSERVABLES:
        out[f"mean_{k}"] = np.asarray(res[f"measurements/Stage0/{k}/mean"])
        out[f"error_{k}"] = np.asarray(res[f"measurements/Stage0/{k}/error"])
    rdm_records(res, ex, out)
    path = os.path.join(HERE, out_name)
    np.savez_compressed(path, **out)
    print(path, settings)


def multidet_case(fn, system, ham_file, wfn_file, case, walker_type, out_name):
    """A seeded snapshot case with a multi-determinant trial: every determinant (upgraded to the
    walker type) and the coefficients; the Hamiltonian tensors are those of the BH closed file."""
    dets, ci, _ = load_nomsd_determinants(os.path.join(fn, "afqmc_inputs", system, wfn_file), walker_type)
    res = H5File(os.path.join(fn, "snapshot_references", system, *case.split("/"), "results.h5"))
    inp = json.loads(res["input_file"])
    ex = inp["execute"]
    settings = dict(seed=inp["seed"], nwalk=ex["num_walkers"], dt=ex["timestep"], steps=ex["steps"],
                    ortho_interval=ex["walker_ortho_interval"], pop_interval=ex["population_control_interval"],
                    measure_interval=ex["measure_interval"], equilibration_steps=ex["equilibration_steps"],
                    num_ranks=int(res["num_ranks"]), walker_type=ex["walker_set"]["walker_type"])
    assert settings["walker_type"] == walker_type
    out = dict(ci_dets=ci, PsiT_dets=np.stack([d["PsiT"] for d in dets]), settings=json.dumps(settings))
    if walker_type == "COLLINEAR":
        out.update(PsiT_up_dets=np.stack([d["PsiT_up"] for d in dets]),
                   PsiT_dn_dets=np.stack([d["PsiT_dn"] for d in dets]))
    for k in OBSERVABLES:
        out[f"mean_{k}"] = np.asarray(res[f"measurements/Stage0/{k}/mean"])
        out[f"error_{k}"] = np.asarray(res[f"measurements/Stage0/{k}/error"])
    rdm_records(res, ex, out)
    path = os.path.join(HERE, out_name)
    np.savez_compressed(path, **out)
    print(path, len(dets), "determinants", settings)


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SAFIRE_REFERENCE_ROOT", "")
    if not src or not os.path.isdir(src):
        sys.exit("usage: make_bh_snapshot.py <SAFIRE source tree> (or set SAFIRE_REFERENCE_ROOT)")
    fn = os.path.join(src, "tests", "functional")
    snapshot_case(fn, "BH", "afqmc_H_rhf_closed.h5", "afqmc_rhf_nomsd.h5", "dense_rhf_basis_closed/rhf_nomsd/closed",
                  "CLOSED", "bh_rhf_closed_snapshot.npz")
    # the same Hamiltonian with a UHF trial (the Hamiltonian tensors are those of the file above)
    snapshot_case(fn, "BH", "afqmc_H_rhf_closed.h5", "afqmc_uhf_nomsd.h5",
                  "dense_rhf_basis_closed/uhf_nomsd/collinear", "COLLINEAR", "bh_uhf_collinear_snapshot.npz",
                  with_hamiltonian=False)
    # the RHF trial upgraded to COLLINEAR walkers (both spins the same orbitals)
    snapshot_case(fn, "BH", "afqmc_H_rhf_closed.h5", "afqmc_rhf_nomsd.h5",
                  "dense_rhf_basis_closed/rhf_nomsd/collinear", "COLLINEAR", "bh_rhf_collinear_snapshot.npz",
                  with_hamiltonian=False)
    # NONCOLLINEAR walkers: the RHF and UHF trials upgraded to spinors, and a GHF trial
    for wfn, name in (("afqmc_rhf_nomsd.h5", "rhf"), ("afqmc_uhf_nomsd.h5", "uhf"), ("afqmc_ghf_nomsd.h5", "ghf")):
        snapshot_case(fn, "BH", "afqmc_H_rhf_closed.h5", wfn, f"dense_rhf_basis_closed/{name}_nomsd/noncollinear",
                      "NONCOLLINEAR", f"bh_{name}_noncollinear_snapshot.npz", with_hamiltonian=False)
    # multi-determinant (CASCI) trials: RHF-based for every walker type, UHF-based, GHF-based
    for wfn, name, wts in (("afqmc_casci_rhf_nomsd.h5", "rcasci_rhf", ("closed", "collinear", "noncollinear")),
                           ("afqmc_casci_uhf_nomsd.h5", "rcasci_uhf", ("collinear", "noncollinear")),
                           ("afqmc_casci_ghf_nomsd.h5", "rcasci_ghf", ("noncollinear",))):
        for wt in wts:
            multidet_case(fn, "BH", "afqmc_H_rhf_closed.h5", wfn, f"dense_rhf_basis_closed/{name}_nomsd/{wt}",
                          wt.upper(), f"bh_{name}_{wt}_snapshot.npz")
    snapshot_case(fn, "Li", "hamil_closed.h5", "rohf_nomsd_polarized.h5",
                  "hamil_closed/rohf_wfn_polarized/collinear", "COLLINEAR", "li_rohf_collinear_snapshot.npz")

    statistical_case(fn, "BH/dense_rhf_basis_closed/rhf_nomsd/closed", "bh_rhf_closed_statistical.json")
    statistical_case(fn, "Li/hamil_closed/rohf_wfn_polarized/collinear", "li_rohf_collinear_statistical.json")


def statistical_case(fn, case, out_name):
    """A statistical reference: its settings (walkers per rank x ranks, steps, equilibration,
    intervals) and the mean / error of the energy observables after equilibration."""
    res = H5File(os.path.join(fn, "statistical_references", *case.split("/"), "results.h5"))
    inp = json.loads(res["input_file"])
    ex = inp["execute"]
    ranks = int(res["num_ranks"])
    nwalk = ex["num_walkers"] if "num_walkers" in ex else ex["n_walkers_per_mpi_task"] * ranks
    stat = dict(seed=inp["seed"], nwalk=nwalk, num_ranks=ranks, dt=ex["timestep"], steps=ex["steps"],
                ortho_interval=ex["walker_ortho_interval"], pop_interval=ex["population_control_interval"],
                measure_interval=ex["measure_interval"], equilibration_steps=ex["equilibration_steps"],
                walker_type=ex["walker_set"]["walker_type"], recorded={})
    for k in ("Energy", "OnebodyEnergy", "ExchangeEnergy", "CoulombEnergy"):
        m, e = complex(res[f"measurements/Stage0/{k}/mean"]), complex(res[f"measurements/Stage0/{k}/error"])
        stat["recorded"][k] = dict(mean=[m.real, m.imag], error=[e.real, e.imag])
    path = os.path.join(HERE, out_name)
    with open(path, "w") as f:
        json.dump(stat, f, indent=1)
    print(path, {k: v for k, v in stat.items() if k != "recorded"})


if __name__ == "__main__":
    main()
