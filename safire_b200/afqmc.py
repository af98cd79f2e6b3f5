"""Python mirror of the reference's AFQMC interfaces, backed by the sm_100a library.

* ``det_ops``-style functions (MixedDensityMatrix, Log_Overlap, Propagate, orthogonalize) and
  ``Real3IndexFactorization`` operations (vbias, vHS, energy) take CUDA tensors (torch) in the
  reference's layouts and call the C ABI on the current torch stream;
* ``AfqmcEngine`` owns one resident system (HamOps + trial + WalkerSet + propagator) and exposes
  Propagate / Orthogonalize / population control / Energy / the run_afqmc loop.

torch is used only for device memory and streams; all arithmetic runs in the library.
"""
import ctypes
import time
import math

import numpy as np

from . import capi
from .capi import check, lib, ptr

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ws(op, nwalk, nmo, nel, nchol=0):
    n = lib().sfq_workspace_size(op, nwalk, nmo, nel, nchol)
    return torch.empty(max(int(n), 1), dtype=torch.uint8, device="cuda")


def _is_cplx(t):
    return t.dtype == torch.complex128


def _need(t, name, dtypes):
    if not t.is_cuda or not t.is_contiguous() or t.dtype not in dtypes:
        raise ValueError(f"{name}: expected a contiguous CUDA tensor of {dtypes}, got {t.dtype} {t.device}")


C128 = (torch.complex128,) if torch else ()
F64 = (torch.float64,) if torch else ()


# ------------------------------------------------------------------------------------------
# det_ops (density_matrix.hpp, propagate.hpp, orthogonalize.hpp)
# ------------------------------------------------------------------------------------------
def MixedDensityMatrix(A, B, compact=True, ovlp=None):
    """det_ops::MixedDensityMatrix(A, B, C, ovlp, compact, herm=true); ovlp accumulates."""
    _need(A, "A", C128 + F64)
    _need(B, "B", C128)
    W, M, N = B.shape
    C = torch.empty((W, N, M) if compact else (W, M, M), dtype=torch.complex128, device="cuda")
    ov = torch.zeros(W, dtype=torch.complex128, device="cuda") if ovlp is None else ovlp
    ws = _ws(capi.OP_MIXED_DENSITY_MATRIX, W, M, N)
    check(lib().sfq_mixed_density_matrix(ptr(A), int(_is_cplx(A)), ptr(B), ptr(C), ptr(ov), W, M, N,
                                         int(compact), ptr(ws), ws.numel(), _stream()))
    return C, ov


def Log_Overlap(A, B, ovlp=None):
    _need(A, "A", C128 + F64)
    _need(B, "B", C128)
    W, M, N = B.shape
    ov = torch.zeros(W, dtype=torch.complex128, device="cuda") if ovlp is None else ovlp
    ws = _ws(capi.OP_LOG_OVERLAP, W, M, N)
    check(lib().sfq_log_overlap(ptr(A), int(_is_cplx(A)), ptr(B), ptr(ov), W, M, N, ptr(ws), ws.numel(),
                                _stream()))
    return ov


def inverse_logdet(A, logdet=None):
    _need(A, "A", C128)
    nb, n, _ = A.shape
    Ainv = torch.empty_like(A)
    ld = torch.zeros(nb, dtype=torch.complex128, device="cuda") if logdet is None else logdet
    check(lib().sfq_inverse_logdet(ptr(A), ptr(Ainv), ptr(ld), nb, n, _stream()))
    return Ainv, ld


def Propagate(SM, P1, V, order=6):
    """det_ops::Propagate<'N'> on CLOSED walkers, in place."""
    _need(SM, "SM", C128)
    _need(P1, "P1", C128 + F64)
    _need(V, "V", C128)
    W, M, N = SM.shape
    ws = _ws(capi.OP_PROPAGATE, W, M, N)
    check(lib().sfq_propagate(ptr(SM), ptr(P1), int(_is_cplx(P1)), ptr(V), W, M, N, order, ptr(ws), ws.numel(),
                              _stream()))
    return SM


def orthogonalize(SM):
    _need(SM, "SM", C128)
    W, M, N = SM.shape
    ws = _ws(capi.OP_ORTHOGONALIZE, W, M, N)
    check(lib().sfq_orthogonalize(ptr(SM), None, W, M, N, ptr(ws), ws.numel(), _stream()))
    return SM


# ------------------------------------------------------------------------------------------
# Real3IndexFactorization (vbias, vHS, energy)
# ------------------------------------------------------------------------------------------
def vbias(G, Lnak, dt, closed=True):
    _need(G, "G", C128)
    _need(Lnak, "Lnak", C128 + F64)
    W = G.shape[0]
    Nc, N, M = Lnak.shape
    v = torch.empty((W, Nc), dtype=torch.complex128, device="cuda")
    check(lib().sfq_vbias(ptr(G), ptr(Lnak), int(_is_cplx(Lnak)), ptr(v), W, N, M, Nc, dt, int(closed), _stream()))
    return v


def vHS(Likn, X, dt):
    _need(Likn, "Likn", F64)
    _need(X, "X", C128)
    M, _, Nc = Likn.shape
    W = X.shape[0]
    V = torch.empty((W, M, M), dtype=torch.complex128, device="cuda")
    check(lib().sfq_vhs(ptr(Likn), ptr(X), ptr(V), W, M, Nc, dt, _stream()))
    return V


def energy(G, haj, Lnak, E0=0.0, addH1=True, addEJ=True, addEXX=True):
    _need(G, "G", C128)
    _need(haj, "haj", C128)
    _need(Lnak, "Lnak", C128 + F64)
    W = G.shape[0]
    Nc, N, M = Lnak.shape
    E = torch.empty((W, 3), dtype=torch.complex128, device="cuda")
    ws = _ws(capi.OP_ENERGY, W, M, N, Nc)
    check(lib().sfq_energy(ptr(E), ptr(G), ptr(haj), ptr(Lnak), int(_is_cplx(Lnak)), E0, W, N, M, Nc, int(addH1),
                           int(addEJ), int(addEXX), ptr(ws), ws.numel(), _stream()))
    return E


def assemble_X(vb, vmf, uniforms=None, seed=0, step=0, vbias_bound=50.0, free_projection=False):
    """X, HW, meanfield_factor from vbias; vb is overwritten with X."""
    _need(vb, "vbias", C128)
    _need(vmf, "vmf", F64)
    W, Nc = vb.shape
    hw = torch.empty(W, dtype=torch.complex128, device="cuda")
    mf = torch.empty(W, dtype=torch.complex128, device="cuda")
    if uniforms is not None:
        _need(uniforms, "uniforms", F64)
    check(lib().sfq_assemble_x(ptr(vb), ptr(vmf), ptr(hw), ptr(mf), ptr(uniforms), seed, step, W, Nc, vbias_bound,
                               int(free_projection), _stream()))
    return vb, hw, mf


def comb(weights, r):
    _need(weights, "weights", F64)
    n = weights.shape[0]
    off = torch.empty(n, dtype=torch.int32, device="cuda")
    check(lib().sfq_comb(ptr(weights), float(r), n, ptr(off), _stream()))
    return off


# ------------------------------------------------------------------------------------------
# Resident engine
# ------------------------------------------------------------------------------------------
class AfqmcEngine:
    """One system resident on one GPU: the drop-in for the objects execute_simulation builds."""

    def __init__(self, system, nwalk, dt=0.005, seed=0, device=0, **params):
        self.M, self.N, self.Nc, self.W = system.M, system.N, system.Nc, nwalk
        self.Mr = getattr(system, "npol", 1) * system.M  # rows of a walker (NONCOLLINEAR spinors: 2M)
        self.dt = dt
        p = capi.system_params(system, nwalk=nwalk, dt=dt, E0=float(system.E0), seed=seed, device=device)
        for k, v in params.items():
            setattr(p, k, v)
        self.params = p
        h = np.ascontiguousarray(system.hcore, dtype=np.float64)
        L = np.ascontiguousarray(system.Likn, dtype=np.float64)
        P = np.ascontiguousarray(system.PsiT, dtype=np.complex128)
        handle = ctypes.c_void_p()
        ci = getattr(system, "ci", None)
        if ci is not None and np.size(ci) > 1:  # multi-determinant trial: PsiT (ndet, rows, cols)
            c = np.ascontiguousarray(ci, dtype=np.complex128)
            check(lib().sfq_engine_create_nomsd(ctypes.byref(handle), ctypes.byref(p), h.ctypes.data, L.ctypes.data,
                                                int(c.size), P.ctypes.data, c.ctypes.data))
        else:
            check(lib().sfq_engine_create(ctypes.byref(handle), ctypes.byref(p), h.ctypes.data, L.ctypes.data,
                                          P.ctypes.data))
        self.h = handle
        self.nbp = 0  # back-propagation ring length (enable_back_propagation)

    def close(self):
        if self.h:
            lib().sfq_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return lib().sfq_engine_stream(self.h)

    def synchronize(self):
        check(lib().sfq_engine_synchronize(self.h))

    # WalkerSet
    def walkers(self):
        SM = np.empty((self.W, self.Mr, self.N), np.complex128)
        pr = np.empty((len(capi.PROPS), self.W), np.complex128)
        check(lib().sfq_engine_get_walkers(self.h, SM.ctypes.data, pr.ctypes.data))
        return SM, {k: pr[i].copy() for i, k in enumerate(capi.PROPS)}

    def set_walkers(self, SM=None, props=None):
        sm = None if SM is None else np.ascontiguousarray(SM, np.complex128)
        pr = None
        if props is not None:
            pr = np.stack([np.asarray(props[k], np.complex128) for k in capi.PROPS])
        check(lib().sfq_engine_set_walkers(self.h, None if sm is None else sm.ctypes.data,
                                           None if pr is None else pr.ctypes.data))

    def properties(self):
        """The property columns alone (WEIGHT, PHASE, ...: W values each), without the Slater matrices."""
        pr = np.empty((len(capi.PROPS), self.W), np.complex128)
        check(lib().sfq_engine_get_walkers(self.h, None, pr.ctypes.data))
        return {k: pr[i].copy() for i, k in enumerate(capi.PROPS)}

    # the sharded walker exchange on device rows (sfq_engine_pack_walkers / unpack_walkers / copy_walkers)
    @property
    def exchange_device(self):
        import torch
        return torch.device("cuda", int(self.params.device))

    def walker_row_elems(self):
        n = int(lib().sfq_engine_walker_row_elems(self.h))
        if n < 0:
            check(-n)
        return n

    def _rows(self, rows, n):
        import torch
        if n and (not isinstance(rows, torch.Tensor) or rows.device != self.exchange_device or not rows.is_contiguous()
                  or rows.dtype != torch.float64 or rows.numel() < n * 2 * self.walker_row_elems()):
            raise capi.SafireError(2, "walker rows: a contiguous float64 tensor of (n, 2 * walker_row_elems()) "
                                      "on the engine's device")
        return ctypes.c_void_p(rows.data_ptr() if n else 0)

    def pack_walkers(self, slots, rows):
        """rows[r] <- walker slots[r] (Slater matrix, then the 8 property values)."""
        sl = np.ascontiguousarray(np.asarray(slots, np.int32).reshape(-1))
        check(lib().sfq_engine_pack_walkers(self.h, sl.ctypes.data, sl.size, self._rows(rows, sl.size)))

    def unpack_walkers(self, slots, rows):
        """walker slots[r] <- rows[r]."""
        sl = np.ascontiguousarray(np.asarray(slots, np.int32).reshape(-1))
        check(lib().sfq_engine_unpack_walkers(self.h, sl.ctypes.data, sl.size, self._rows(rows, sl.size)))

    def copy_walkers(self, pairs, normalize=True):
        """Every weight to w / |w| (normalize), then walker dst <- walker src for (src, dst) in pairs."""
        pr = np.ascontiguousarray(np.asarray(pairs, np.int32).reshape(-1, 2))
        check(lib().sfq_engine_copy_walkers(self.h, pr.ctypes.data, len(pr), int(bool(normalize))))

    def walker_buffer(self):
        rows = np.empty((self.W, self.Mr * self.N + 11), np.complex128)
        check(lib().sfq_engine_export_walker_buffer(self.h, rows.ctypes.data))
        return rows

    # Wavefunction / Propagator
    def energy(self, seed_pseudo=False):
        E = np.empty((self.W, 3), np.complex128)
        check(lib().sfq_engine_energy(self.h, int(seed_pseudo), E.ctypes.data))
        return E

    def init(self):
        """execute.cpp:172-184: Energy, seedPseudoEnergy, Eshift = averageEnergy."""
        self.energy(seed_pseudo=True)
        return self.averages()[1]

    def propagate(self, Eshift, step, uniforms=None):
        check(lib().sfq_engine_propagate(self.h, float(Eshift), int(step), None if uniforms is None else
                                         ctypes.c_void_p(ptr(uniforms))))

    def propagate_host(self, Eshift, step, uniforms_host=None, props_out=None):
        check(lib().sfq_engine_propagate_host(self.h, float(Eshift), int(step),
                                              None if uniforms_host is None else ctypes.c_void_p(ptr(uniforms_host)),
                                              None if props_out is None else ctypes.c_void_p(ptr(props_out))))

    def orthogonalize(self):
        check(lib().sfq_engine_orthogonalize(self.h))

    def population_control(self, call=0, uniform=None):
        """population_control: the comb draws Philox(seed, call), or takes `uniform` in [0, 1)."""
        if uniform is None:
            check(lib().sfq_engine_population_control(self.h, int(call)))
        else:
            check(lib().sfq_engine_population_control_uniform(self.h, float(uniform)))

    def averages(self):
        pe, e, tw = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib().sfq_engine_averages(self.h, ctypes.byref(pe), ctypes.byref(e), ctypes.byref(tw)))
        return pe.value, e.value, tw.value

    def measure(self):
        o = np.empty(10, np.float64)
        check(lib().sfq_engine_measure(self.h, o.ctypes.data))
        keys = ("Energy", "OnebodyEnergy", "ExchangeEnergy", "CoulombEnergy", "TotalWeight")
        return {k: complex(o[2 * i], o[2 * i + 1]) for i, k in enumerate(keys)}

    def _rdm_buffers(self):
        nspin = 2 if self.params.walker_type == capi.WALKER_COLLINEAR else 1
        M = self.M
        n2 = M * (2 * M - 1) - (M * (M - 1) // 2 if self.params.walker_type == capi.WALKER_CLOSED else 0)
        return np.empty((nspin, self.Mr, self.Mr), np.complex128), np.empty(n2, np.complex128)

    def measure_mixed_rdms(self):
        """MixedEstimator's OneRDM and DiagonalTwoRDM of the current walkers (sfq_engine_measure_rdm)."""
        one, two = self._rdm_buffers()
        check(lib().sfq_engine_measure_rdm(self.h, one.ctypes.data, two.ctypes.data))
        return {"MixedEstimator/OneRDM": one, "MixedEstimator/DiagonalTwoRDM": two}

    def enable_back_propagation(self, nbp):
        """Keep the fields and weight factors of the last nbp steps per walker (resize_bp)."""
        check(lib().sfq_engine_enable_back_propagation(self.h, int(nbp)))
        self.nbp = int(nbp)

    def bp_anchor(self):
        check(lib().sfq_engine_bp_anchor(self.h))

    def measure_bp_rdms(self, nsteps, ortho_interval=10, path_restoration=True):
        """BackPropEstimator's OneRDM and DiagonalTwoRDM over the last nsteps (sfq_engine_measure_bp_rdm)."""
        one, two = self._rdm_buffers()
        check(lib().sfq_engine_measure_bp_rdm(self.h, int(nsteps), int(ortho_interval), int(bool(path_restoration)),
                                              one.ctypes.data, two.ctypes.data))
        pre = f"BackPropEstimator/Steps={int(nsteps)}"
        return {f"{pre}/OneRDM": one, f"{pre}/DiagonalTwoRDM": two}

    def _obs_buffers(self, two_rdm, spin_corr, pair_maps):
        M = self.M
        ns = 2 if self.params.walker_type == capi.WALKER_COLLINEAR else 1
        two = np.empty((ns + 1, M, M, M, M), np.complex128) if two_rdm else None
        spin = np.empty((2, M * (M + 1) // 2), np.complex128) if spin_corr else None
        maps = None if pair_maps is None else np.ascontiguousarray(np.asarray(pair_maps, np.int32))
        pair = None if maps is None else np.empty((len(maps), len(maps), M, M), np.complex128)
        p = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        return (two, spin, maps, pair), (p(two), p(spin), 0 if maps is None else len(maps), p(maps), p(pair))

    @staticmethod
    def _obs_dict(pre, two, spin, pair):
        out = {}
        if two is not None:
            out[f"{pre}/TwoRDM"] = two
        if spin is not None:
            out[f"{pre}/SpinCorr"] = spin
        if pair is not None:
            out[f"{pre}/PairCorr"] = pair
        return out

    def measure_observables(self, two_rdm=True, spin_corr=True, pair_maps=None):
        """MixedEstimator's TwoRDM, SpinCorr and PairCorr (pair_maps (npair, nmo): each orbital's
        partner, negative for none) of the current walkers (sfq_engine_measure_observables)."""
        (two, spin, _, pair), args = self._obs_buffers(two_rdm, spin_corr, pair_maps)
        check(lib().sfq_engine_measure_observables(self.h, *args))
        return self._obs_dict("MixedEstimator", two, spin, pair)

    def measure_bp_observables(self, nsteps, ortho_interval=10, path_restoration=True, two_rdm=True, spin_corr=True,
                               pair_maps=None):
        """BackPropEstimator's TwoRDM, SpinCorr and PairCorr over the last nsteps."""
        (two, spin, _, pair), args = self._obs_buffers(two_rdm, spin_corr, pair_maps)
        check(lib().sfq_engine_measure_bp_observables(self.h, int(nsteps), int(ortho_interval),
                                                      int(bool(path_restoration)), *args))
        return self._obs_dict(f"BackPropEstimator/Steps={int(nsteps)}", two, spin, pair)

    # TimeEvolvedBPEstimator (sfq_engine_*_te_*): the operators evolve through the back-propagation ring
    def enable_time_evolved_bp(self):
        check(lib().sfq_engine_enable_time_evolved_bp(self.h))

    def te_anchor(self):
        check(lib().sfq_engine_te_anchor(self.h))

    def te_evolve(self, nsteps):
        check(lib().sfq_engine_te_evolve(self.h, int(nsteps)))

    def measure_te_rdms(self, steps, restore_steps):
        """The one-body and folded diagonal two-body RDMs of the evolved operators, the weights
        restored over restore_steps (0: none)."""
        one, two = self._rdm_buffers()
        check(lib().sfq_engine_measure_te_rdm(self.h, int(restore_steps), one.ctypes.data, two.ctypes.data))
        pre = f"TimeEvolvedBP/Steps={int(steps)}"
        return {f"{pre}/OneRDM": one, f"{pre}/DiagonalTwoRDM": two}

    def measure_te_observables(self, steps, restore_steps, two_rdm=True, spin_corr=True, pair_maps=None):
        (two, spin, _, pair), args = self._obs_buffers(two_rdm, spin_corr, pair_maps)
        check(lib().sfq_engine_measure_te_observables(self.h, int(restore_steps), *args))
        return self._obs_dict(f"TimeEvolvedBP/Steps={int(steps)}", two, spin, pair)

    def run_with_streams(self, steps, Eshift, field_uniforms, comb_uniform, ortho_interval=10, pop_interval=10,
                         equilibration_steps=100, measure_interval=10, relax=None, step0=0, mixed_interval=None,
                         bp_steps=None, bp_ortho_interval=None, path_restoration=True, observables=None,
                         te_steps=None, te_extra_path_restoration=False):
        """run_afqmc's step loop (run_afqmc.cpp:69-104) with the caller's random streams at the
        reference's two injection points: field_uniforms(n) returns the n = nwalk * nchol uniforms
        of a step (walker-major, assemble_X's sampleUniformFields) and comb_uniform() the comb's
        uniform (population_control.hpp:41-42).  Given the reference's own generators it replays
        a reference run.  Every measurement records EnergyEstimator::measure's observables
        (EnergyEstimator.h:51-100), every mixed_interval steps the mixed estimator's RDMs, and with
        bp_steps the back-propagated ones; observables (keyword arguments of measure_observables) adds
        TwoRDM, SpinCorr and PairCorr to both estimators; te_steps runs TimeEvolvedBPEstimator's schedule
        (TimeEvolvedBPEstimator.hpp:199-220) instead of bp_steps.
        Returns (Eshift, {observable: list of bins})."""
        if relax is None:
            relax = 1 - math.exp(-10.0 / equilibration_steps) if equilibration_steps > 1 else 1.0
        series = {}
        if bp_steps:  # BackPropEstimator's schedule (BackPropEstimator.hpp:150-168): anchored at step0 - 1
            bp_steps = sorted(int(k) for k in bp_steps)
            self.enable_back_propagation(bp_steps[-1])
            bp_pos = step0 - 1
        if te_steps:
            te_steps = sorted(int(k) for k in te_steps)
            self.enable_back_propagation(te_steps[-1])
            self.enable_time_evolved_bp()
            te_pos = step0 - 1
        for step in range(step0, step0 + steps):
            u = np.ascontiguousarray(np.asarray(field_uniforms(self.W * self.Nc), np.float64).reshape(self.W, self.Nc))
            self.propagate_host(Eshift, step, uniforms_host=u)
            if step % ortho_interval == 0:
                self.orthogonalize()
            if step % pop_interval == 0:
                self.population_control(uniform=float(comb_uniform()))
            if step >= equilibration_steps:
                if step % measure_interval == 0:
                    m = self.measure()
                    _, pr = self.walkers()
                    w, ov = pr["WEIGHT"], pr["OVLP"]
                    aw = np.abs(w)
                    m["Overlap"] = complex(np.sum(np.exp(ov) * w) / np.sum(w))
                    m["ProjectionTime"] = (step + 1) * self.dt
                    m["EffectiveNumWalkers"] = float(np.sum(aw) ** 2 / np.sum(aw * aw))
                    m["Phase"] = complex(np.sum(w) / np.sum(aw))
                    for k, v in m.items():
                        series.setdefault(k, []).append(v)
                if mixed_interval and step % mixed_interval == 0:
                    for k, v in self.measure_mixed_rdms().items():
                        series.setdefault(k, []).append(v)
                    if observables:
                        for k, v in self.measure_observables(**observables).items():
                            series.setdefault(k, []).append(v)
                if bp_steps:
                    if step - bp_pos in bp_steps:
                        for k, v in self.measure_bp_rdms(step - bp_pos, bp_ortho_interval or ortho_interval,
                                                         path_restoration).items():
                            series.setdefault(k, []).append(v)
                        if observables:
                            for k, v in self.measure_bp_observables(step - bp_pos, bp_ortho_interval or ortho_interval,
                                                                    path_restoration, **observables).items():
                                series.setdefault(k, []).append(v)
                    if step - bp_pos >= bp_steps[-1]:
                        self.bp_anchor()
                        bp_pos = step
                if te_steps:
                    bp = step - te_pos
                    if bp in te_steps:
                        i = te_steps.index(bp)
                        self.te_evolve(bp - (te_steps[i - 1] if i > 0 else 0))
                        restore = bp * (2 if te_extra_path_restoration else 1) if path_restoration else 0
                        for k, v in self.measure_te_rdms(bp, restore).items():
                            series.setdefault(k, []).append(v)
                        if observables:
                            for k, v in self.measure_te_observables(bp, restore, **observables).items():
                                series.setdefault(k, []).append(v)
                    if bp >= te_steps[-1]:
                        self.te_anchor()
                        te_pos = step
            else:
                Eshift += relax * (self.averages()[0] - Eshift)
        return Eshift, series

    def run(self, steps, Eshift, ortho_interval=10, pop_interval=10, equilibration_steps=100, measure_interval=10,
            relax=0.0, step0=0, max_meas=4096, steer=False):
        rp = capi.RunParams(steps, ortho_interval, pop_interval, equilibration_steps, measure_interval, relax, step0,
                            int(steer))
        es = ctypes.c_double(Eshift)
        meas = np.zeros((max_meas, 10), np.float64)
        nm = ctypes.c_int()
        check(lib().sfq_engine_run(self.h, ctypes.byref(rp), ctypes.byref(es), meas.ctypes.data, max_meas,
                                   ctypes.byref(nm)))
        return es.value, meas[:nm.value]

    def run_block(self, steps, Eshift, ortho_interval=10, pop_interval=10, equilibration_steps=100,
                  measure_interval=10, relax=0.0, step0=0, steer=False):
        """The same loop as run(), device-resident and replayed from a CUDA graph (sfq_engine_block)."""
        rp = capi.RunParams(steps, ortho_interval, pop_interval, equilibration_steps, measure_interval, relax, step0,
                            int(steer))
        es = ctypes.c_double(Eshift)
        meas = np.zeros((64, 10), np.float64)
        nm = ctypes.c_int()
        check(lib().sfq_engine_block(self.h, ctypes.byref(rp), ctypes.byref(es), meas.ctypes.data, 64,
                                     ctypes.byref(nm)))
        return es.value, meas[:nm.value]

    def block_async(self, steps, Eshift, ortho_interval=10, pop_interval=10, equilibration_steps=100,
                    measure_interval=10, relax=0.0, step0=0, steer=False):
        rp = capi.RunParams(steps, ortho_interval, pop_interval, equilibration_steps, measure_interval, relax, step0,
                            int(steer))
        check(lib().sfq_engine_block_async(self.h, ctypes.byref(rp), float(Eshift)))

    def block_query(self):
        rc = lib().sfq_engine_block_query(self.h)
        if rc < 0:
            check(-rc)
        return rc == 1

    def block_result(self):
        es = ctypes.c_double()
        meas = np.zeros((64, 10), np.float64)
        nm = ctypes.c_int()
        check(lib().sfq_engine_block_result(self.h, ctypes.byref(es), meas.ctypes.data, 64, ctypes.byref(nm)))
        return es.value, meas[:nm.value]

    def autotune(self, repeats=9):
        """Time every built tile width of each mixed product on this engine and keep the fastest
        (sfq_engine_autotune); returns the Tiles record (choice and per-product times)."""
        t = capi.Tiles()
        check(lib().sfq_engine_autotune(self.h, int(repeats), ctypes.byref(t)))
        return t

    def tiles(self):
        t = capi.Tiles()
        check(lib().sfq_engine_tiles(self.h, ctypes.byref(t)))
        return t.choice()

    def set_tiles(self, g_bn=0, vbias_bn=0, vhs_bn=0, taylor_half=0, p1_bn=0, vbias_ksplit=0):
        t = capi.Tiles(g_bn, vbias_bn, vhs_bn, taylor_half, p1_bn, vbias_ksplit)
        check(lib().sfq_engine_set_tiles(self.h, ctypes.byref(t)))

    def footprint(self):
        b = ctypes.c_size_t()
        check(lib().sfq_engine_footprint(self.h, ctypes.byref(b)))
        return b.value

    def profile(self, enable=True):
        check(lib().sfq_engine_profile(self.h, int(enable)))

    def phase_times(self):
        ms = np.zeros(len(capi.PHASES), np.float64)
        cnt = np.zeros(len(capi.PHASES), np.int32)
        check(lib().sfq_engine_phase_times(self.h, ms.ctypes.data, cnt.ctypes.data, len(capi.PHASES)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(capi.PHASES)}

    def info(self):
        inf = capi.EngineInfo()
        check(lib().sfq_engine_info(self.h, ctypes.byref(inf)))
        return inf

    def fetch(self, name, shape, dtype):
        """Copy one of the engine's resident device arrays (by EngineInfo field) to the host."""
        inf = self.info()
        out = np.empty(shape, dtype)
        check(lib().sfq_memcpy(out.ctypes.data, getattr(inf, name), out.nbytes, 2, None))
        return out


class EngineGroup:
    """Several resident engines (systems of any sizes) advanced together: one block of every member
    per call, all members' blocks captured as branches of one CUDA graph (sfq_group_*)."""

    MAX_MEAS = 64

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (ctypes.c_void_p * len(self.engines))(*[e.h for e in self.engines])
        h = ctypes.c_void_p()
        check(lib().sfq_group_create(ctypes.byref(h), arr, len(self.engines)))
        self.h = h
        self.lanes = 0
        self.fused = False

    def close(self):
        if self.h:
            lib().sfq_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _params(self, steps, ortho_interval, pop_interval, equilibration_steps, measure_interval, relax, step0,
                steer):
        n = len(self.engines)
        step0 = np.broadcast_to(np.asarray(step0, np.uint64), (n,))
        relax = np.broadcast_to(np.asarray(relax, np.float64), (n,))
        rps = (capi.RunParams * n)()
        for i in range(n):
            rps[i] = capi.RunParams(steps, ortho_interval, pop_interval, equilibration_steps, measure_interval,
                                    float(relax[i]), int(step0[i]), int(steer))
        return rps

    def block_async(self, steps, Eshift, ortho_interval=10, pop_interval=10, equilibration_steps=100,
                    measure_interval=10, relax=0.0, step0=0, steer=False):
        rps = self._params(steps, ortho_interval, pop_interval, equilibration_steps, measure_interval, relax, step0,
                           steer)
        es = np.ascontiguousarray(np.broadcast_to(np.asarray(Eshift, np.float64), (len(self.engines),)))
        check(lib().sfq_group_block_async(self.h, rps, es.ctypes.data))

    def block_query(self):
        rc = lib().sfq_group_block_query(self.h)
        if rc < 0:
            check(-rc)
        return rc == 1

    def block_result(self, raise_errors=True):
        """(Eshift per member, status per member, list of measurement arrays per member)"""
        n = len(self.engines)
        es = np.zeros(n, np.float64)
        status = np.zeros(n, np.int32)
        meas = np.zeros((n, self.MAX_MEAS, 10), np.float64)
        nm = np.zeros(n, np.int32)
        rc = lib().sfq_group_block_result(self.h, es.ctypes.data, status.ctypes.data, meas.ctypes.data,
                                          self.MAX_MEAS, nm.ctypes.data)
        if raise_errors:
            check(rc)
        return es, status, [meas[i, :nm[i]] for i in range(n)]

    def run_block(self, steps, Eshift, **kw):
        self.block_async(steps, Eshift, **kw)
        return self.block_result()

    def set_lanes(self, lanes):
        """Schedule: `lanes` chains run side by side, members of a chain in turn (0: one per member)."""
        check(lib().sfq_group_set_lanes(self.h, int(lanes)))
        self.lanes = int(lanes)

    def set_fused(self, on=True):
        """Fused schedule (int8-slice members on one block schedule): the members' steps stage by
        stage, each stage's tensor-core products of all members as one grouped launch."""
        check(lib().sfq_group_set_fused(self.h, 1 if on else 0))
        self.fused = bool(on)

    def _schedule(self, c):
        if c == "fused":
            self.set_fused(True)
        else:
            self.set_fused(False)
            self.set_lanes(c)

    def tune_lanes(self, steps, Eshift, step0=0, candidates=("fused", 1, 2, 3, 4, 6, 8, 0), **kw):
        """Schedule autotuner: run real blocks with each schedule ("fused" where every member runs an
        int8-slice precision, else a lane count), one to capture its graph and one timed, and keep
        the fastest.  Returns (Eshift, next step0, {schedule: seconds per block})."""
        times = {}
        es = Eshift
        int8 = all(e.params.precision in (capi.PRECISION_INT8X3, capi.PRECISION_INT8X2) for e in self.engines)
        for c in candidates:
            if c == "fused" and not int8:
                continue
            if c != "fused" and c > len(self.engines):
                continue
            self._schedule(c)
            es, _st, _m = self.run_block(steps, es, step0=step0, **kw)
            step0 += steps
            t0 = time.perf_counter()
            es, _st, _m = self.run_block(steps, es, step0=step0, **kw)
            times[c] = time.perf_counter() - t0
            step0 += steps
        self._schedule(min(times, key=times.get))
        return es, step0, times
