#!/usr/bin/env python
"""Throughput of the lDGA ladder chain on B200.

One step = the whole hot path for one parameter point of the 3D simple-cubic workload
(eps_k = -2t sum cos k_i, N_k = 32^3 -> 969 irreducible q, beta = 20, U = 1.5, Nnu = 40, Nw = 41):
lattice G and its transform -> bubble chi0 -> Bethe-Salpeter (m, d) -> F_m, lambda_0 -> lambda_m
correction (device Newton) -> EoM Sigma_ladder(lambda_m) -> mu fit, G_ladder, energies.
metric = (q, w)-points per second = N_q * N_w per step, summed over ranks (each rank runs its own
seeded parameter point: weak scaling, no data-path collective).

  value  device-resident inputs; per-step CUDA-event time on the stream the library launches on
  e2e    the same chain through the C ABI from pinned HOST buffers (inputs copied in, Sigma_ladder,
         chi_m, chi_d, lambda, mu, energies copied out inside the timed region)
  --impl reference  the CPU restatement (oracle/) of the reference algorithm on all host cores

L2 is flushed (256 MiB write) before every timed step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(cfg=3, dim=3, ns=32, beta=20.0, U=1.5, n_iv=20, n_iw=20)
WORKLOAD_NAME = "3D sc Nk=32^3 (969 irreducible q), beta=20, U=1.5, Nnu=40, Nw=41, lambda_m"
# the other single-point configurations, selectable with --cfg (the chain is the lambda_m chain for all)
CFG_NAMES = {
    1: "2D sq Nk=16^2 (45 irreducible q), beta=10, U=1, Nnu=20, Nw=21, lambda_m",
    2: "2D sq Nk=64^2 (561 irreducible q), beta=30, U=2, Nnu=60, Nw=61, lambda_dm",
    3: WORKLOAD_NAME,
}
METRIC = "(q,w)-points/s"
PREC_NAMES = {"fp64inv": 0, "fp64": 1, "mixed": 2}
REF_BUDGET_S = 120.0
REF_DM_STEPS = 10
# DRAM bytes per BSE matrix (Nnu = 40) from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum of
# one launch): the FP64 LU on 3D 16^3 (6765 matrices) and the MIXED preconditioned solve on 3D 32^3 (39 729)
BSE_DRAM_BYTES_PER_MATRIX = 5423872 / 6765
BSE_ITER_DRAM_BYTES_PER_MATRIX = (26807808 + 100608) / 39729
BSE_TILE = 8   # rows per diagonal block of the LU kernels at Nnu = 40


def BSE_EXEC_CMACS(n: int, t: int = BSE_TILE) -> float:
    """Complex multiply-adds the LU kernels execute for one matrix: the forward elimination of
    [B | 1] (step k updates the rows of its diagonal block and below, except row k, in the columns
    right of k), the block back substitution (N^2/2) and the FP64 backward-error product (N^2)."""
    fwd = sum((n - t * (k // t) - 1) * (n - k) for k in range(n))
    return fwd + n * n / 2.0 + n * n


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--prec", default="mixed", choices=list(PREC_NAMES),
                    help="BSE precision mode (mixed: FP32 preconditioner with FP64 residuals, results verified "
                         "to FP64 backward error 1e-14; fp64: the FP64 LU)")
    ap.add_argument("--tune-file", default=None,
                    help="load BSE configuration choices (ldga_tune_save format) instead of autotuning")
    ap.add_argument("--bse-config", default=None,
                    help="use this BSE configuration (a name ldga_bse_config_name reports, e.g. iter8x2dm:3) for the "
                         "workload's box size and precision instead of autotuning")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip timing the same chain in FP64 mode (mixed runs report mixed / FP64)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the oracle chain (the CPU baseline and the accuracy check against it)")
    ap.add_argument("--no-stage-events", action="store_true",
                    help="time the chain without the per-stage CUDA events inside its graph (no stage times)")
    ap.add_argument("--ns", type=int, default=None, help="smaller k-grid (points per axis) for profiling captures")
    ap.add_argument("--out", default=None, help="also write the JSON line to this file")
    ap.add_argument("--workload", default="chain", choices=["chain", "batch", "adjoint"],
                    help="chain: the 3D 32^3 point (default); batch: the uneven 64-point (U, beta) scan on 2D 32^2; "
                         "adjoint: the chain's vector-Jacobian product (ldga_chain_vjp) against its forward "
                         "(ldga_chain_m) on 2D 48^2, Nnu=40, Nw=41")
    ap.add_argument("--points", type=int, default=64, help="points of the batch workload")
    ap.add_argument("--shard", default="points", choices=["points", "omega"],
                    help="points: every rank runs its own parameter point (weak scaling, the default); omega: "
                         "the ranks split one point's bosonic frequencies (strong scaling; the chain runs stage "
                         "by stage with one all-reduce of chi and one of Sigma_ladder)")
    ap.add_argument("--cfg", type=int, default=3, choices=[1, 2, 3],
                    help="single-point configuration of the chain workload (3: the headline 3D 32^3 point)")
    ap.add_argument("--lambda", dest="lam", default=None, choices=["m", "dm"],
                    help="lambda correction of the chain workload (default: dm for --cfg 2, m otherwise)")
    ap.add_argument("--input", default=None,
                    help="a readConfig TOML file: run the chain workload on that DMFT impurity input "
                         "(e.g. tests/golden/b1u2_plain.toml) instead of a synthetic configuration")
    return ap.parse_args()


def workload_input(args, rank: int = 0):
    """(input, workload name, data label) of the chain workload."""
    if args.input:
        import ladderdga_b200 as L
        from ladderdga_b200 import inputs as I
        _, mP, sP, env, kgs = L.readConfig(args.input)
        inp = I.load_impurity_input(env.inputVars, kgs[0], mP, sP)
        nq = L.gen_kGrid(*kgs[0]).kMult.size
        name = (f"DMFT input {os.path.basename(env.inputVars)}: {inp.dim}D sc Nk={inp.ns}^{inp.dim} "
                f"({nq} irreducible q), beta={inp.beta:g}, U={inp.U:g}, Nnu={2 * inp.n_iv}, "
                f"Nw={2 * inp.n_iw + 1}, shift={inp.shift}, lambda_m")
        return inp, name, f"DMFT impurity file {os.path.basename(env.inputVars)} (read by readConfig)"
    from ladderdga_b200 import synthetic as S
    over = {"ns": args.ns} if args.ns else {}
    name = CFG_NAMES[args.cfg]
    if lam_type(args) != ("dm" if args.cfg == 2 else "m"):
        name = name.rsplit(", ", 1)[0] + f", lambda_{lam_type(args)}"
    return S.config_input(args.cfg, point=rank, **over), name, "synthetic"


def lam_type(args) -> str:
    return args.lam or ("dm" if args.cfg == 2 and not args.input else "m")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ----------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        return self.summary()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, n in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ----------------------------------------------------------------------------------------------
# CPU baseline: the oracle restatement of the reference algorithm on the host cores
# ----------------------------------------------------------------------------------------------
def oracle_chain(inp, lambda_type="m"):
    """The oracle's chain on the workload (with the lambda_m correction, or none): (outputs, seconds)."""
    from oracle import ldga_ref as R
    R.set_workers(os.cpu_count() or 1)
    t0 = time.perf_counter()
    ref = R.run_chain(inp, lambda_type=lambda_type)
    return ref, time.perf_counter() - t0


def cpu_chain_seconds(inp, lt: str = "m") -> float:
    if lt == "m":
        return oracle_chain(inp, "m")[1]
    # lambda_dm: the oracle's chain up to lambda_0 and its own lambda_dm Newton, capped at REF_DM_STEPS
    # iterations (at ~0.4 s a residual and 3 residuals an iteration the full 500-step budget of the
    # reference's newton_right would take minutes per step): a lower bound of the step's time
    from oracle import ldga_ref as R
    ref, t = oracle_chain(inp, None)
    t0 = time.perf_counter()
    R.lambda_dm_correction(ref["chi_m"], ref["gamma_m"], ref["chi_d"], ref["gamma_d"], ref["lambda0"], ref["h"],
                           nsteps=REF_DM_STEPS)
    return t + time.perf_counter() - t0


def cpu_baseline(t: float, points: int) -> dict:
    return {"value": points / t, "unit": METRIC, "cores": os.cpu_count() or 1, "kind": "port",
            "sample": f"one full chain of the workload ({t:.1f} s): NumPy/SciPy FP64 restatement of the "
                      "reference algorithm (oracle/ldga_ref.py), scipy.fft workers and OpenBLAS threads = all cores"}


# ----------------------------------------------------------------------------------------------
# accuracy of the timed step against the FP64 oracle
# ----------------------------------------------------------------------------------------------
# Elementwise relative errors divide by max(|ref|, ERR_FLOOR * max|ref|): an entry that cancels to
# ~1e-6 of the array's largest one carries FP64 rounding of the large terms (~1e-16 of them), so
# 1e-10 elementwise is the bar FP64 arithmetic itself can meet down to that floor.
ERR_FLOOR = 1e-6


def rel_err(a, b) -> dict:
    a, b = np.asarray(a), np.asarray(b)
    d = np.abs(a - b)
    m = float(np.max(np.abs(b))) if b.size else 0.0
    m = m if m > 0 else 1e-300
    e = d / np.maximum(np.abs(b), ERR_FLOOR * m)
    i = int(np.argmax(e))
    return {"elementwise": float(e.flat[i]), "normwise": float(d.max() / m),
            "worst": [int(x) for x in np.unravel_index(i, b.shape)]}


def chi_err(dev_chi, ref, r: str, beta: float, U: float) -> dict:
    """chi_r(q, w) = Re sum_nu y_nu / beta^2 sums terms of both signs; where they cancel, no FP64
    evaluation is more accurate than the terms' magnitude allows.  'componentwise' divides each error by
    that magnitude, sum_nu |y_nu| / beta^2 with y = gamma chi0 (1 + s U chi) from the oracle (the
    reference's conditioning of the sum); 'elementwise' divides by |chi| with the usual floor."""
    s = 1.0 if r == "m" else -1.0
    chi_r = ref[f"chi_{r}"].data
    y = ref[f"gamma_{r}"] * ref["chi0"] * (1.0 + s * U * chi_r)[:, None, :]
    scale = np.abs(y).sum(axis=1) / beta ** 2
    d = np.abs(np.asarray(dev_chi) - chi_r)
    e = d / np.maximum(scale, 1e-300)
    i = int(np.argmax(e))
    out = rel_err(dev_chi, chi_r)
    out["componentwise"] = float(e.flat[i])
    out["componentwise_worst"] = [int(x) for x in np.unravel_index(i, chi_r.shape)]
    return out


def array_errors(chain, ref) -> dict:
    """chi0, gamma_m, gamma_d and lambda0 elementwise, chi_m and chi_d componentwise (chi_err), from the
    handle's device copies."""
    from ladderdga_b200 import _lib
    ctx, h = chain.ctx, chain.h
    nq, nnu, nw = ctx.Nq, ctx.Nnu, ctx.Nw

    def get(what, ch=0, real=False):
        out = np.empty((nq, nw), order="F") if real else _lib.cplx_out((nq, nnu, nw))
        ctx.call("ldga_get", what, ch, _lib.ptr(out))
        return out

    beta, U = h.mP.β, h.mP.U
    return {"floor": f"elementwise denominators max(|oracle|, {ERR_FLOOR:g} max|oracle|)",
            "chi0": rel_err(get(_lib.GET_CHI0), ref["chi0"]),
            "chi_m": chi_err(get(_lib.GET_CHI, _lib.CH_M, True), ref, "m", beta, U),
            "chi_d": chi_err(get(_lib.GET_CHI, _lib.CH_D, True), ref, "d", beta, U),
            "gamma_m": rel_err(get(_lib.GET_GAMMA, _lib.CH_M), ref["gamma_m"]),
            "gamma_d": rel_err(get(_lib.GET_GAMMA, _lib.CH_D), ref["gamma_d"]),
            "lambda0": rel_err(get(_lib.GET_LAMBDA0), ref["lambda0"])}


def accuracy_dm(chain, ref, scal) -> dict:
    """Errors of the handle's last lambda_dm chain against the oracle on the same input.  The oracle's
    own lambda_dm Newton takes minutes on this box (one residual = an FFT EoM, a mu fit and the energies,
    ~0.4 s), so the device's root (lambda_m, lambda_d) is put into the ORACLE's residual (conditions_new.jl
    residual_vals): |F| measures how well it solves the reference's equations, Sigma_ladder is compared
    at that root, and the mu fit, G_ladder and energies are compared from the oracle's Sigma_ladder
    ('isolated').  ref: the oracle chain without lambda correction; returns (errors, seconds of one
    oracle residual)."""
    from oracle import ldga_ref as R
    from ladderdga_b200 import _lib
    ctx, h = chain.ctx, chain.h
    errs = array_errors(chain, ref)
    lm, ld = scal[0], scal[8]
    numax = chain.dm_numax
    S_dev = _lib.cplx_out((ctx.Nq, numax))
    ctx.call("ldga_get", _lib.GET_SIGMA, 0, _lib.ptr(S_dev))
    hr = ref["h"]
    t0 = time.perf_counter()
    n, mu, ek, ep1, ep2, lhs_c1, Sr, Gr = R.lambda_dm_residual(np.array([lm, ld]), ref["chi_m"], ref["gamma_m"],
                                                               ref["chi_d"], ref["gamma_d"], ref["lambda0"], hr,
                                                               numax, {"mu": hr.mP.mu})
    t_res = time.perf_counter() - t0
    rhs_c1 = hr.mP.n / 2 * (1 - hr.mP.n / 2)
    ctx.call("ldga_set_sigma", _lib.ptr(_lib.as_fc(Sr)), numax)
    G = _lib.cplx_out((ctx.Nq, ctx.Nf))
    mu_d, ek_d, ep_d, n_d = (C.c_double() for _ in range(4))
    ctx.call("ldga_g_ladder", None, 0, 1, h.mP.μ, C.byref(mu_d), _lib.ptr(G), C.byref(ek_d), C.byref(ep_d),
             C.byref(n_d))
    iso = {"G_ladder": rel_err(G, Gr), "mu_abs": abs(mu_d.value - mu),
           "E_kin_rel": abs(ek_d.value - ek) / max(1.0, abs(ek)), "E_pot1_rel": abs(ep_d.value - ep1) / max(1.0, abs(ep1))}
    errs["at_device_root"] = {
        "lambda_m": lm, "lambda_d": ld, "converged": bool(scal[6]),
        "oracle_residual": [lhs_c1 - rhs_c1, ep1 - ep2],
        "Sigma_ladder": rel_err(S_dev, Sr), "mu_abs": abs(scal[1] - mu), "isolated": iso}
    checked = [errs[k]["elementwise"] for k in ("chi0", "gamma_m", "gamma_d", "lambda0")]
    checked += [errs[k]["componentwise"] for k in ("chi_m", "chi_d")]
    checked += [errs["at_device_root"]["Sigma_ladder"]["elementwise"], errs["at_device_root"]["mu_abs"],
                iso["G_ladder"]["elementwise"], iso["mu_abs"], iso["E_kin_rel"], iso["E_pot1_rel"]]
    errs["max_checked"] = float(max(checked))
    errs["root_residual_ok"] = bool(math.hypot(lhs_c1 - rhs_c1, ep1 - ep2) <= 1e-8)
    errs["checked"] = ("chi0, gamma, lambda0 elementwise; chi componentwise; Sigma_ladder and mu at the device's "
                       "root; G_ladder, mu, energies isolated from the oracle's Sigma_ladder there; the root itself "
                       "to the Newton's atol 1e-8 in the oracle's residual")
    errs["within_1e-10"] = bool(errs["max_checked"] <= 1e-10 and errs["root_residual_ok"])
    return errs, t_res


def accuracy(chain, ref, lam_dev: float) -> dict:
    """Errors of the handle's last chain step against the oracle chain on the same input.

    chi0, gamma_m, gamma_d and lambda0 elementwise; chi_m, chi_d componentwise (chi_err).  lambda_m of
    this workload is not a parity quantity (the reference's newton_right runs into the poles of f, see
    `lambda_m`), so the lambda-dependent stages are checked at the ORACLE's lambda_m: 'isolated' gives
    each stage the oracle's inputs (EoM from the oracle's chi, gamma, lambda0; mu fit, G_ladder and the
    energies from the oracle's Sigma_ladder) and measures that stage alone; 'propagated' runs them on
    the device's own upstream results, whose differences the near-pole chi_lambda = chi/(1 + lambda chi)
    amplifies by `amplification` = max |1/(1 + lambda chi)|.  (This overwrites the handle's arrays.)"""
    from oracle import ldga_ref as R
    from ladderdga_b200 import _lib
    ctx, h = chain.ctx, chain.h
    nq, nnu, nw, numax = ctx.Nq, ctx.Nnu, ctx.Nw, chain.numax
    beta, U = h.mP.β, h.mP.U

    def get(what, ch=0, real=False):
        out = np.empty((nq, nw), order="F") if real else _lib.cplx_out((nq, nnu, nw))
        ctx.call("ldga_get", what, ch, _lib.ptr(out))
        return out

    res = ref["result"]
    errs = array_errors(chain, ref)
    lam = float(res.lam_m)

    def downstream():
        S = _lib.cplx_out((nq, numax))
        ctx.call("ldga_eom", lam, 0.0, numax, 1, h.χloc_m_sum, _lib.ptr(S))
        return S

    def g_ladder():
        G = _lib.cplx_out((nq, ctx.Nf))
        mu, ek, ep, n = (C.c_double() for _ in range(4))
        ctx.call("ldga_g_ladder", None, 0, 1, h.mP.μ, C.byref(mu), _lib.ptr(G), C.byref(ek), C.byref(ep),
                 C.byref(n))
        return G, mu.value, ek.value, ep.value

    def stage_errs(S, G, mu, ek, ep):
        return {"Sigma_ladder": rel_err(S, res.Sigma_ladder), "G_ladder": rel_err(G, res.G_ladder),
                "mu_abs": abs(mu - res.mu), "E_kin_rel": abs(ek - res.EKin) / max(1.0, abs(res.EKin)),
                "E_pot1_rel": abs(ep - res.EPot_p1) / max(1.0, abs(res.EPot_p1))}

    # propagated: the device's own chi, gamma, lambda0 at the oracle's lambda_m
    S = downstream()
    prop = stage_errs(S, *g_ladder())
    cm = ref["chi_m"].data
    prop["amplification"] = float(np.max(np.abs(1.0 / (1.0 + lam * cm))))
    # isolated: each stage from the oracle's inputs
    ctx.call("ldga_set_chi", _lib.CH_M, _lib.ptr(np.asfortranarray(ref["chi_m"].data)))
    ctx.call("ldga_set_chi", _lib.CH_D, _lib.ptr(np.asfortranarray(ref["chi_d"].data)))
    ctx.call("ldga_set_gamma", _lib.CH_M, _lib.ptr(_lib.as_fc(ref["gamma_m"])))
    ctx.call("ldga_set_gamma", _lib.CH_D, _lib.ptr(_lib.as_fc(ref["gamma_d"])))
    ctx.call("ldga_set_lambda0", _lib.ptr(_lib.as_fc(ref["lambda0"])))
    S_iso = downstream()
    ctx.call("ldga_set_sigma", _lib.ptr(_lib.as_fc(res.Sigma_ladder)), numax)
    iso = stage_errs(S_iso, *g_ladder())
    errs["at_oracle_lambda_m"] = {"lambda_m": lam, "isolated": iso, "propagated": prop}
    # lambda_m itself: both values, and how well each solves the oracle's f(l) = sum_kw chi_l - rhs
    rh, cmT = ref["h"], ref["chi_m"]
    rhs = 2 * rh.imp_density - R.sum_kw(rh.kG, ref["chi_d"])

    def f(l):
        return R.sum_kw(rh.kG, cmT, transform=lambda x: R.chi_lambda(x, l)) - rhs

    def scale(l):
        return max(1.0, R.sum_kw(rh.kG, cmT, transform=lambda x: np.abs(R.chi_lambda(x, l))))

    neg = cm[cm < 0]
    errs["lambda_m"] = {
        "device": lam_dev, "oracle": lam, "abs_diff": abs(lam_dev - lam),
        "device_root_residual": abs(f(lam_dev)) / scale(lam_dev), "oracle_root_residual": abs(f(lam)) / scale(lam),
        "f_at_0": f(0.0), "df_c1_at_0": R.sum_kw(rh.kG, cmT, transform=lambda x: R.dchi_lambda(x, 0.0)),
        "first_pole": float(1.0 / np.max(-neg)) if neg.size else None,
        "note": "newton_right's df carries the chi tail constants (df_c1 > 0 at 0 while f(0) < 0), so the "
                "iteration walks right into the poles of f at lambda >= first_pole, where each iterate depends "
                "on the rounding of the sums: every root it can land on solves f = 0, but which one is not a "
                "parity quantity"}
    checked = [errs[k]["elementwise"] for k in ("chi0", "gamma_m", "gamma_d", "lambda0")]
    checked += [errs[k]["componentwise"] for k in ("chi_m", "chi_d")]
    checked += [iso["Sigma_ladder"]["elementwise"], iso["G_ladder"]["elementwise"], iso["mu_abs"],
                iso["E_kin_rel"], iso["E_pot1_rel"]]
    errs["max_checked"] = float(max(checked))
    errs["checked"] = ("chi0, gamma, lambda0 elementwise; chi componentwise; Sigma_ladder, G_ladder, mu, "
                       "energies isolated at the oracle's lambda_m")
    errs["within_1e-10"] = bool(errs["max_checked"] <= 1e-10)
    return errs


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    inp, wname, data = workload_input(args)
    from oracle import ldga_ref as R
    points = R.gen_kGrid(inp.kgrid_kind, inp.ns).Nq * (2 * inp.n_iw + 1)
    # one step is a whole chain (about 10 s on 8 cores): the warm-up is capped at one chain and the
    # timed steps stop once REF_BUDGET_S seconds are spent, so the arm ends within a few minutes
    for _ in range(min(args.warmup, 1)):
        cpu_chain_seconds(inp, lam_type(args))
    ts = []
    t_start = time.perf_counter()
    while len(ts) < args.steps and (not ts or time.perf_counter() - t_start < REF_BUDGET_S):
        ts.append(cpu_chain_seconds(inp, lam_type(args)))
    ms = 1000.0 * float(np.mean(ts))
    value = points / (ms / 1000.0)
    what = ("full chain(s)" if lam_type(args) == "m" else
            f"chain(s) with the lambda_dm Newton capped at {REF_DM_STEPS} iterations (a lower bound of the step)")
    sample = (f"{len(ts)} {what} of the workload after {min(args.warmup, 1)} warm-up chain(s) "
              f"(steps capped by a {REF_BUDGET_S:.0f} s budget); NumPy/SciPy FP64 restatement of the reference "
              "algorithm (oracle/ldga_ref.py), scipy.fft workers and OpenBLAS threads = all cores")
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": len(ts),
            "steps_requested": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": data,
            "impl": "reference",
            "config": {"workload": wname, "global_batch": 1, "l2": "inputs resident in host memory"},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": os.cpu_count() or 1, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if args.out:
        open(args.out, "w").write(json.dumps(line) + "\n")
    return 0


# ----------------------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------------------
class Chain:
    """The device chain for one parameter point, driven through the C ABI."""

    def __init__(self, inp, prec: int, device: int, stream=None, lam_type: str = "m"):
        import torch
        import ladderdga_b200 as L
        self.L, self.torch = L, torch
        self.inp = inp
        self.lam_type = lam_type
        self.h = L.setup_synthetic(inp, precision=prec, device=device)
        self.ctx = self.h.ctx
        self.lib = self.ctx.lib
        self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        self.ctx.call("ldga_set_stream", C.c_void_p(self.stream.cuda_stream))
        h = self.h
        dev = torch.device("cuda", device)

        def cplx(a):
            return np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(-1, order="F")).view(np.float64)

        host = {"sigma_loc": cplx(h.Σ_loc), "gamma_m": cplx(h.Γ_m), "gamma_d": cplx(h.Γ_d),
                "chi_loc_m": cplx(h.χDMFT_m), "gimp": cplx(h.gImp)}
        self.h2d_bytes = sum(v.nbytes for v in host.values())
        # pinned host copies (e2e) and device-resident copies (value)
        self.pin = {k: torch.from_numpy(v).pin_memory() for k, v in host.items()}
        self.dev = {k: torch.from_numpy(v).to(dev) for k, v in host.items()}
        self.n_sigma = len(h.Σ_loc)
        self.n_gimp = len(h.gImp)
        nq, nw, numax = self.ctx.Nq, self.ctx.Nw, h.sP.n_iν
        self.numax = numax
        self.out_sigma = torch.empty(nq * numax * 2, dtype=torch.float64).pin_memory()
        self.out_chi_m = torch.empty(nq * nw, dtype=torch.float64).pin_memory()
        self.out_chi_d = torch.empty(nq * nw, dtype=torch.float64).pin_memory()
        self.d2h_bytes = (self.out_sigma.numel() + self.out_chi_m.numel() + self.out_chi_d.numel()) * 8 + 5 * 8
        if lam_type == "dm":   # Sigma_ladder (at most n_iv frequencies) and 7 scalars come back
            self.d2h_bytes = self.out_sigma.numel() * 8 + 7 * 8
        self.points = nq * nw
        self.dm_evals = 0

    def io(self, src: dict, outputs: bool, sc):
        """This point's ldga_chain_io (ldga_batch_chain_m)."""
        from ladderdga_b200 import _lib
        p = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
        return _lib.ChainIO(p(src["sigma_loc"]), self.n_sigma, p(src["gamma_m"]), p(src["gamma_d"]),
                            p(src["chi_loc_m"]), p(src["gimp"]), self.n_gimp, self.h.imp_density, self.h.χloc_m_sum,
                            p(self.out_sigma) if outputs else None, p(self.out_chi_m) if outputs else None,
                            p(self.out_chi_d) if outputs else None, C.addressof(sc))

    def step_dm(self, src: dict, outputs: bool):
        """One parameter point through the lambda_dm chain of the C ABI: ldga_gloc -> ldga_bubble ->
        ldga_bse (m, d) -> ldga_F_from_chi -> ldga_lambda0 -> ldga_lambda_dm (the reference's 2-D
        newton_right on the host, every residual an EoM + mu fit + energies on the device).
        Scalars as ldga_chain_m's, [6] = converged, [8] = lambda_d."""
        from ladderdga_b200 import _lib
        p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        ctx = self.ctx
        ctx.call("ldga_gloc", p(src["sigma_loc"]), self.n_sigma, None)
        ctx.call("ldga_bubble", None)
        ctx.call("ldga_bse", _lib.CH_M, p(src["gamma_m"]), None, None, None)
        ctx.call("ldga_bse", _lib.CH_D, p(src["gamma_d"]), None, None, None)
        ctx.call("ldga_F_from_chi", p(src["chi_loc_m"]), p(src["gimp"]), self.n_gimp, None)
        ctx.call("ldga_lambda0", None, None)
        lm, ld, conv, nu = C.c_double(), C.c_double(), C.c_int32(), C.c_int32()
        out7 = (C.c_double * 7)()
        st = self.lib.ldga_lambda_dm(ctx.h, self.h.χloc_m_sum, -1, 1e-4, 1e-8, 500, C.byref(lm), C.byref(ld),
                                     C.byref(conv), out7, C.byref(nu), p(self.out_sigma) if outputs else None, None)
        if st != _lib.LDGA_ERR_NOCONV:
            ctx.check(st)
        ev = C.c_int32()
        ctx.call("ldga_lambda_dm_evals", C.byref(ev))
        self.dm_evals, self.dm_numax = ev.value, nu.value
        n, mu, ek, ep1, ep2, pp1, pp2 = list(out7)
        return [lm.value, mu, ek, ep1, ep2, pp2, float(conv.value), n, ld.value]

    def step(self, src: dict, outputs: bool, graph: bool = True):
        """One parameter point through ldga_chain_m (captured once in a CUDA graph, then replayed)."""
        if self.lam_type == "dm":
            return self.step_dm(src, outputs)
        p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        sc = (C.c_double * 8)()
        self.ctx.call("ldga_chain_m", p(src["sigma_loc"]), self.n_sigma, p(src["gamma_m"]), p(src["gamma_d"]),
                      p(src["chi_loc_m"]), p(src["gimp"]), self.n_gimp, self.h.imp_density, self.h.χloc_m_sum,
                      int(graph), p(self.out_sigma) if outputs else None, p(self.out_chi_m) if outputs else None,
                      p(self.out_chi_d) if outputs else None, sc)
        return list(sc)


TUNE_FILE = None
BSE_CONFIG = None


def tune(chain) -> str:
    """Untimed: run the bubble, let the autotuner pick the BSE configuration for this box size and
    precision mode (both channels' inputs) -- or load the choices of --tune-file -- and return its
    name."""
    ctx = chain.ctx
    ctx.call("ldga_bubble", None)
    import ladderdga_b200 as L
    if BSE_CONFIG and ctx.precision == BSE_CONFIG[0]:
        import tempfile
        with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
            f.write(f"bse {ctx.Nnu} {ctx.precision} {BSE_CONFIG[1]}\n")
        try:
            L.tune_load(f.name)
        finally:
            os.unlink(f.name)
        got = chain.lib.ldga_bse_config_name(ctx.Nnu, ctx.precision, -1)
        if not got or got.decode() != BSE_CONFIG[1]:
            raise SystemExit(f"--bse-config {BSE_CONFIG[1]}: not a configuration of Nnu={ctx.Nnu}, mode {ctx.precision}")
    elif TUNE_FILE:
        L.tune_load(TUNE_FILE)
    else:
        for t in ("m", "d"):
            L.autotune_bse(chain.h, t, reps=3)
    name = chain.lib.ldga_bse_config_name(ctx.Nnu, ctx.precision, -1)
    return name.decode() if name else "pivoted"


def newton_period(chain):
    """The λm Newton of the last step rerun alone (newton_right's nsteps 100, atol 1e-13): the
    iterations it reports and where its state began to repeat (iteration, period), from which on
    whole periods are skipped."""
    try:
        chid = C.c_double()
        chain.ctx.call("ldga_sum_kw", 1, 0.0, 0, C.byref(chid))
        lam, its, per = C.c_double(), C.c_int32(), (C.c_int32 * 2)()
        chain.ctx.call("ldga_lambda_m_newton", 2 * chain.h.imp_density - chid.value, 100, 1e-13, C.byref(lam),
                       C.byref(its), per)
        return {"lambda_m": lam.value, "iterations": its.value, "repeat_at": per[0], "period": per[1],
                "executed": per[0] + (its.value - per[0]) % per[1] if per[1] else its.value}
    except Exception as e:  # reported, not fatal: the bench line stands without it
        return {"error": str(e)}


STAGE_BSE_MASK = 1 << 2   # LDGA_STAGE_BSE


def stage_breakdown(chain, steps: int) -> dict:
    """Per-stage device time of the chain (ms per step) from `steps` untimed replays with every
    stage's events in the graph; profiling is off afterwards."""
    chain.ctx.call("ldga_profile", 1)
    for _ in range(2):                      # the first call re-captures the graph with the events
        chain.step(chain.dev, False)
    stage_times(chain)
    for _ in range(steps):
        chain.step(chain.dev, False)
    st = stage_times(chain)
    chain.ctx.call("ldga_profile", 0)
    return {k: v[0] / steps for k, v in st.items() if v[1]}


def stage_times(chain):
    from ladderdga_b200._lib import STAGES
    ms = (C.c_double * 10)()
    cnt = (C.c_int32 * 10)()
    chain.ctx.call("ldga_stage_times", ms, cnt)
    return {STAGES[i]: (ms[i], cnt[i]) for i in range(10)}


def measure_fp64_peak(device: int, n: int = 8192, reps: int = 5) -> float:
    """FP64 throughput of a cuBLAS DGEMM (n^3, the FP64 tensor path) on this GPU in TFLOP/s: the
    measured denominator of the FP64-bound kernels' roofline (the driver's peaks have no FP64 entry)."""
    import torch
    dev = torch.device("cuda", device)
    g = torch.Generator(device=dev).manual_seed(0)
    a = torch.rand(n, n, dtype=torch.float64, device=dev, generator=g)
    b = torch.rand(n, n, dtype=torch.float64, device=dev, generator=g)
    c = torch.empty_like(a)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.matmul(a, b, out=c)
    e1.record()
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 * reps / t / 1e12


def fp64_peak(peaks: dict, sm_mhz: float):
    if peaks.get("fp64_tflops"):
        return peaks["fp64_tflops"], peaks.get("fp64_source", "measured FP64 throughput")
    return (148 * 64 * 2 * sm_mhz * 1e6 / 1e12,
            f"nominal 64 FP64 FMA/clk/SM x 148 SMs x {sm_mhz:.0f} MHz (no FP64 figure measured)")


def roofline(stages: dict, chain, peaks: dict, sweeps=None, steps: int = 1) -> dict:
    """Dominant stage of the step and its roofline (algorithmic work per launch / CUDA-event time)."""
    name = max(stages, key=lambda k: stages[k][0])
    tot, cnt = stages[name]
    t = tot / max(cnt, 1) / 1e3   # seconds per launch
    nq, nnu, nw = chain.ctx.Nq, chain.ctx.Nnu, chain.ctx.Nw
    hbm = peaks.get("hbm_gbs", 6650.0)
    if name == "bse":
        # algorithmic work per (q, w) matrix: the reference's complex LU + inverse (zgetrf + zgetri,
        # 8 N^3 real flops) plus the sums (8 N^2); a step solves both channels, N_q N_w matrices each,
        # in one launch (the preconditioned solve) or two
        chans = 2.0 * steps / max(cnt, 1)
        flops = chans * nq * nw * (8.0 * nnu**3 + 8.0 * nnu**2)
        ach = flops / t / 1e12
        # what the kernel executes: elimination of [B | 1] alone (BSE_EXEC_CMACS complex multiply-adds)
        exe = chans * nq * nw * 8.0 * BSE_EXEC_CMACS(nnu) / t / 1e12
        sm_mhz = peaks.get("sm_max_mhz", 1965.0)
        cfg = chain.lib.ldga_bse_config_name(nnu, chain.ctx.precision, -1)
        cfg = cfg.decode() if cfg else ""
        if cfg.startswith("iter"):
            # MIXED preconditioned solve: the FP64 residual passes set the bound.  Executed work from
            # the kernel's own counters (ldga_bse_sweeps): every warp evaluates the residual of its q
            # in lockstep, 8 N^2 + 8 N FP64 flops per q and pass (6 N^2 + 8 N on the FP64 tensor
            # path, whose complex product takes three real products); the FP32 corrections 8 N^2 each.
            peak, peak_src = fp64_peak(peaks, sm_mhz)
            qpw = {"iter": 8, "iter8": 4, "iter8x2": 8, "iter8x2tc": 8, "iter8x2dm": 8,
                   "iter8x2dm2": 8}.get(cfg.split(":")[0], 8)
            nprod = 2.0 if "dm2" in cfg else 1.0   # the second-order correction: two TF32 products a pass
            passes, warps = sweeps if sweeps else (0, 1)
            prod = 6.0 if "dm" in cfg else 8.0
            f64 = passes * qpw * (prod * nnu**2 + 8.0 * nnu) / max(cnt, 1)
            f32 = nprod * (passes - warps) * qpw * 8.0 * nnu**2 / max(cnt, 1)
            exe = f64 / t / 1e12
            kname = ("k_bse_iter (FP32 group inverse; FP64 residual on the FP64 tensor path, mma.sync m8n8k4, "
                     "three real products per complex tile; second-order correction C r - C (dD C r), two TF32 "
                     "tensor-core products a pass)" if "dm2" in cfg else
                     "k_bse_iter (FP32 group inverse; FP64 residual on the FP64 tensor path, mma.sync m8n8k4, "
                     "three real products per complex tile; FP32 product on tensor cores, mma.sync TF32)"
                     if "dm" in cfg else
                     "k_bse_iter (FP32 group inverse, FP64 residual passes, FP32 product on tensor cores: "
                     "mma.sync TF32)" if "tc" in cfg else "k_bse_iter (FP32 group inverse, FP64 residual passes)")
            return {"kernel": kname, "bound": "fp64",
                    "achieved": exe, "peak": peak, "unit": "TFLOP/s", "frac": exe / peak,
                    "work": (f"executed FP64 flops of the residual passes ({prod:.0f} N^2 + 8 N per q and pass, "
                             "warps in lockstep), counted by the kernel"),
                    "passes_per_warp": passes / max(warps, 1),
                    "fp32_tflops": f32 / t / 1e12,
                    "reference_formulation_tflops": ach,
                    "reference_formulation_frac_of_bf16": ach / peaks.get("bf16_tflops", 1590.0),
                    "channels_per_launch": chans,
                    "traffic": BSE_ITER_DRAM_BYTES_PER_MATRIX * chans * nq * nw if nnu == 40 else None,
                    "traffic_source": ("ncu dram__bytes_read+write of one launch on 3D 32^3 (39 729 matrices)"
                                       if nnu == 40 else "no capture at this Nnu"),
                    "peak_source": peak_src}
        # bound: FP32 (mixed) / FP64 CUDA-core pipes, nominal B200 rates at the measured max clock
        # the FP32 eliminations (MIXED's lu32 / warp configurations) or the FP64 LU (FP64 mode, and
        # MIXED where the autotuner found it fastest)
        fp = "fp32" if cfg.startswith(("lu32", "warp")) else "fp64"
        lanes = 128 if fp == "fp32" else 64
        peak = 148 * lanes * 2 * sm_mhz * 1e6 / 1e12
        peak_src = (f"nominal {lanes} {fp.upper()} FMA/clk/SM x 148 SMs x {sm_mhz:.0f} MHz (the CUDA-core pipe, "
                    "not HBM or tensor cores, bounds this kernel)")
        if fp == "fp64":
            peak, peak_src = fp64_peak(peaks, sm_mhz)
        kname = ("k_bse_warp32 (FP32 LU per warp + FP64 refinement)" if cfg.startswith("warp") else
                 "k_bse_lu32 (FP32 LU + FP64 refinement)" if fp == "fp32" else "k_bse_lu (FP64 LU)")
        kname += f" [{cfg}]"
        return {"kernel": kname, "bound": fp, "achieved": ach, "peak": peak,
                "unit": "TFLOP/s", "frac": ach / peak,
                "work": "8 N^3 + 8 N^2 flops per matrix (the reference's LU + inverse formulation)",
                "executed": {"tflops": exe, "frac": exe / peak,
                             "work": "flops of the LU solve of [B | 1], its back substitution and the "
                                     "backward-error check (one pass; refinement sweeps not counted)"},
                "channels_per_launch": chans,
                "traffic": BSE_DRAM_BYTES_PER_MATRIX * chans * nq * nw if nnu == 40 else None,
                "traffic_source": ("ncu dram__bytes_read+write of one FP64 launch on 3D 16^3 (6765 matrices, "
                                   "802 B each), scaled by the matrix count" if nnu == 40 else
                                   "no capture at this Nnu"),
                "peak_source": peak_src}
    # HBM-bound stages: algorithmic bytes per launch
    byts = {
        "bubble": (nq * (nnu + 1) * 16 * 2 + nq * nnu * nw * 16),
        "eom_forward": nq * chain.numax * nw * (3 * 16 + 2 * 8) + nq * chain.numax * 16,
        "gloc": nq * chain.ctx.Nf * 16 * 2,
    }.get(name, nq * nnu * nw * 16)
    ach = byts / t / 1e9
    return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "traffic": None,
            "peak_source": peaks.get("source", "measured hbm_gbs (MEASURED_PEAKS.json)")}


def run_omega_sharded(args):
    """One parameter point's λm chain with its ω range split over the ranks (parallel.py): every
    step is bubble -> BSE (m, d) -> λ₀ on this rank's block, one all-reduce of χ_m and χ_d, the λm
    Newton, this block's Σ_ladder part, one all-reduce of Σ_ladder, the μ fit and the energies.
    Strong scaling: value = the point's (q, ω) units / the slowest rank's step time (CUDA events on
    the handle's stream around each step; the step's library calls return after their work)."""
    import torch
    import ladderdga_b200 as L
    from ladderdga_b200 import parallel as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    group = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    inp, wname, data = workload_input(args, 0)          # every rank: the same point
    if lam_type(args) != "m":
        raise SystemExit("--shard omega runs the lambda_m chain")
    h = L.setup_synthetic(inp, precision=PREC_NAMES[args.prec], device=local)
    stream = torch.cuda.current_stream(local)
    h.ctx.call("ldga_set_stream", C.c_void_p(stream.cuda_stream))
    stages = P.HandleStages(h)
    points = h.ctx.Nq * h.ctx.Nw
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    n0 = C.c_int64()
    res = None
    for _ in range(max(args.warmup, 3)):
        res = P.λm_chain_omega_sharded(stages, group)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    h.ctx.call("ldga_launch_count", C.byref(n0))
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        res = P.λm_chain_omega_sharded(stages, group)
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    n1 = C.c_int64()
    h.ctx.call("ldga_launch_count", C.byref(n1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = float(np.mean(times))
    if world > 1:
        from ladderdga_b200.parallel import max_over_ranks
        ms = max_over_ranks(ms, device=torch.device("cuda", local))
    if rank == 0:
        line = {"metric": METRIC, "value": points / (ms / 1e3), "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64+f32" if args.prec == "mixed" else "f64", "data": data,
                "impl": "ours", "precision_mode": args.prec,
                "config": {"workload": wname, "global_batch": 1, "seq_len": None, "parallelism": f"omega{world}",
                           "l2": "flushed (256 MiB write) before each step", "points_per_step": points,
                           "omega_block": list(res["block"])},
                "gpu_launches": int(n1.value - n0.value),
                "result": {"lambda_m": res["lambda_m"], "mu": res["mu"], "E_kin": res["E_kin"],
                           "E_pot1": res["E_pot1"], "newton_iterations": res["newton_iterations"]},
                "clocks": clk}
        print(json.dumps(line), flush=True)
        if args.out:
            with open(args.out, "w") as f:
                f.write(json.dumps(line) + "\n")
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    inp, wname, data = workload_input(args, rank)
    lt = lam_type(args)
    chain = Chain(inp, PREC_NAMES[args.prec], local, lam_type=lt)
    bse_config = tune(chain)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        peaks = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback (no MEASURED_PEAKS.json)"}
    try:
        peaks["fp64_tflops"] = measure_fp64_peak(local)
        peaks["fp64_source"] = "cuBLAS DGEMM 8192^3 (FP64 tensor path) measured in this run"
    except Exception as e:  # reported, not fatal: the roofline then states the nominal figure
        peaks["fp64_error"] = str(e)

    def timed(src, outputs):
        times = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(chain.stream)
            chain.step(src, outputs)
            b.record(chain.stream)
            b.synchronize()
            times.append(a.elapsed_time(b))
        return times

    # Inside the timed region only the BSE launches (the dominant kernel, whose duration the roofline
    # needs) are bracketed by CUDA events: every event is a node of the chain's graph and delays it.
    # The per-stage breakdown comes from a separate, untimed pass with every stage's events.
    chain.ctx.call("ldga_profile_stages", 0 if args.no_stage_events else STAGE_BSE_MASK)
    for _ in range(max(args.warmup, 3)):
        scal = chain.step(chain.dev, False)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    stage_times(chain)
    n0 = C.c_int64()
    chain.ctx.call("ldga_launch_count", C.byref(n0))
    chain.ctx.call("ldga_bse_sweeps", None, None)
    t_dev = timed(chain.dev, False)
    sp, sw = C.c_int64(), C.c_int64()
    chain.ctx.call("ldga_bse_sweeps", C.byref(sp), C.byref(sw))
    n1 = C.c_int64()
    chain.ctx.call("ldga_launch_count", C.byref(n1))
    stages = stage_times(chain)
    for _ in range(max(args.warmup, 3)):
        chain.step(chain.pin, True)
    t_e2e = timed(chain.pin, True)
    torch.cuda.synchronize()
    clk = clocks.stop()
    breakdown = stage_breakdown(chain, min(args.steps, 10))
    newton = newton_period(chain) if lt == "m" else {"lambda_dm_residual_evaluations": chain.dm_evals}
    # the oracle's chain on the same input: the CPU baseline's timing and the reference values of
    # the accuracy check (rank 0 at N = 1 only)
    oref, t_cpu, errors, errors64 = None, None, None, None
    if world == 1 and not args.no_cpu_baseline:
        if lt == "m":
            oref, t_cpu = oracle_chain(inp, "m")
            errors = accuracy(chain, oref, scal[0])
        else:
            # the oracle's chain up to lambda_0, then one residual of its lambda_dm at the device's root;
            # the CPU time of a whole step counts that residual as many times as the device's Newton
            # evaluated its own
            oref, t_cpu = oracle_chain(inp, None)
            scal = chain.step(chain.dev, False)
            errors, t_res = accuracy_dm(chain, oref, scal)
            # the reference's FiniteDiff Jacobian evaluates f(x) once more per Newton iteration (3 device
            # residuals an iteration plus the one at the root)
            n_ref = chain.dm_evals + (chain.dm_evals - 1) // 3
            t_cpu_sample = (t_cpu, t_res, n_ref)
            t_cpu = t_cpu + n_ref * t_res
    ms = float(np.mean(t_dev))
    ms_e2e = float(np.mean(t_e2e))
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms, ms_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e = float(t[0]), float(t[1])
    value = world * chain.points / (ms / 1e3)
    e2e = world * chain.points / (ms_e2e / 1e3)
    launches = int(n1.value - n0.value)
    fp64_cmp = None
    if args.prec == "mixed" and world == 1 and not args.no_fp64_compare:
        # the same chain with the FP64 LU, same timing: the mixed / FP64 ratio of the headline metric
        c64 = Chain(inp, PREC_NAMES["fp64"], local, lam_type=lt)
        cfg64 = tune(c64)
        c64.ctx.call("ldga_profile_stages", 0 if args.no_stage_events else STAGE_BSE_MASK)
        for _ in range(max(args.warmup, 3)):
            scal64 = c64.step(c64.dev, False)
        torch.cuda.synchronize()
        stage_times(c64)
        tr = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(c64.stream)
            c64.step(c64.dev, False)
            b.record(c64.stream)
            b.synchronize()
            tr.append(a.elapsed_time(b))
        rst = stage_times(c64)
        c64.ctx.call("ldga_profile", 0)
        brk64 = stage_breakdown(c64, min(args.steps, 10))
        if oref is not None:
            errors64 = accuracy(c64, oref, scal64[0]) if lt == "m" else accuracy_dm(c64, oref, scal64)[0]
        ms64 = float(np.mean(tr))
        bse64 = rst["bse"][0] / args.steps
        bse_mx = stages["bse"][0] / args.steps or float("nan")
        fp64_cmp = {"ms_per_step": ms64, "value": chain.points / (ms64 / 1e3), "bse_config": cfg64,
                    "bse_ms_per_step": bse64, "mixed_over_fp64": ms64 / ms,
                    "bse_mixed_over_fp64": bse64 / bse_mx,
                    "stages_ms_per_step": brk64}
        if errors64 is not None:
            fp64_cmp["errors"] = errors64
    if rank == 0:
        rl = (roofline(stages, chain, peaks, (sp.value, sw.value), args.steps) if any(v[1] for v in stages.values())
              else {"note": "no stage events (--no-stage-events)"})
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if args.prec != "mixed" else "f64+f32",
                "data": data, "impl": "ours", "precision_mode": args.prec,
                "config": {"workload": wname, "global_batch": world, "seq_len": None,
                           "parallelism": f"replicas{world}", "l2": "flushed (256 MiB write) before each step",
                           "points_per_step_per_gpu": chain.points, "bse_config": bse_config},
                "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": chain.h2d_bytes,
                        "d2h_bytes_per_step": chain.d2h_bytes, "ms_per_step": ms_e2e,
                        "path": "C ABI (ldga_*) from pinned host buffers"},
                "roofline": rl,
                "stages_ms_per_step": breakdown,
                "stages_note": "untimed pass with CUDA events around every stage (the events delay the graph; "
                               "the timed region brackets only the BSE launches)",
                "gpu_launches": launches,
                "result": {"lambda_m": scal[0], "mu": scal[1], "E_kin": scal[2], "E_pot1": scal[3],
                           **({"lambda_d": scal[8], "converged": bool(scal[6]), "E_pot2": scal[4], "PP_p2": scal[5]}
                              if lt == "dm" else {}),
                           "newton_iterations": scal[6], "newton_rerun": newton},
                "clocks": clk}
        if errors is not None:
            line["errors"] = errors
        if fp64_cmp is not None:
            line["fp64_compare"] = fp64_cmp
        if t_cpu is not None:
            line["cpu_baseline"] = cpu_baseline(t_cpu, chain.points)
            if lt == "dm":
                tc, tr, nr = t_cpu_sample
                line["cpu_baseline"]["sample"] = (
                    f"the oracle's chain up to lambda_0 ({tc:.1f} s) and one residual of its lambda_dm Newton "
                    f"({tr:.2f} s), counted {nr} times (the residual evaluations the reference's Newton makes on the "
                    "device's trajectory): NumPy/SciPy FP64 restatement of the reference algorithm (oracle/ldga_ref.py), "
                    "scipy.fft workers and OpenBLAS threads = all cores")
        print(json.dumps(line), flush=True)
        if args.out:
            open(args.out, "w").write(json.dumps(line) + "\n")
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


ADJ_NAME = ("2D sq Nk=48^2 (325 irreducible q), beta=20, U=1.5, Nnu=40, Nw=41: forward = the lambda_m chain "
            "(ldga_chain_m), adjoint = dL/dGamma_m, dL/dGamma_d, dL/dSigma_loc of L = sum |Sigma_ladder|^2 at the "
            "chain's lambda_m (ldga_chain_vjp)")


def run_adjoint(args):
    """The adjoint's cost against the forward chain on the same point (time ratio, lower is better)."""
    import torch
    from ladderdga_b200 import synthetic as S
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    inp = S.config_input(4)
    chain = Chain(inp, PREC_NAMES[args.prec], local)
    bse_config = tune(chain)
    ctx, stream = chain.ctx, chain.stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(args.warmup, 3)):
        scal = chain.step(chain.dev, True)
    torch.cuda.synchronize()
    lam_m = scal[0]
    nq, nnu, nw, numax = ctx.Nq, ctx.Nnu, ctx.Nw, chain.numax
    dev = torch.device("cuda", local)
    sig = chain.out_sigma.to(dev)                                   # Sigma_ladder [Nq, numax] (re, im)
    sbar = 2.0 * sig                                                # dL/dSigma for L = sum |Sigma|^2
    n_sigma = chain.n_sigma
    gm_bar = torch.empty(nnu * nnu * nw * 2, dtype=torch.float64, device=dev)
    gd_bar = torch.empty_like(gm_bar)
    sl_bar = torch.empty(n_sigma * 2, dtype=torch.float64, device=dev)
    nf = C.c_int32()
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    def adjoint():
        ctx.call("ldga_chain_vjp", p(sbar), lam_m, 0.0, numax, 1, p(gm_bar), p(gd_bar), n_sigma, p(sl_bar), None,
                 C.byref(nf))

    def timed(fn):
        times = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b))
        return times

    for _ in range(max(args.warmup, 3)):
        adjoint()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    n0 = C.c_int64()
    ctx.call("ldga_launch_count", C.byref(n0))
    t_fwd = timed(lambda: chain.step(chain.dev, False))
    n1 = C.c_int64()
    ctx.call("ldga_launch_count", C.byref(n1))
    t_adj = timed(adjoint)
    n2 = C.c_int64()
    ctx.call("ldga_launch_count", C.byref(n2))
    clk = clocks.stop()
    fwd, adj = float(np.mean(t_fwd)), float(np.mean(t_adj))
    line = {"metric": "adjoint / forward time", "value": adj / fwd, "unit": "ratio", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": adj, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "ours",
            "precision_mode": args.prec,
            "config": {"workload": ADJ_NAME, "global_batch": 1, "l2": "flushed (256 MiB write) before each step",
                       "points_per_step_per_gpu": chain.points, "bse_config": bse_config},
            "forward_ms": fwd, "adjoint_ms": adj,
            "forward_points_per_s": chain.points / (fwd / 1e3), "adjoint_points_per_s": chain.points / (adj / 1e3),
            "adjoint_flagged_solves": nf.value,
            "gpu_launches": {"forward": int(n1.value - n0.value) // args.steps,
                             "adjoint": int(n2.value - n1.value) // args.steps, "unit": "per step"},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    if args.out:
        open(args.out, "w").write(json.dumps(line) + "\n")
    return 0


BATCH_NAME = ("uneven batch: {n} points of 2D sc Nk=32^2 (153 irreducible q), U ~ U[0.5,3], beta in {{5,10,20,40}}, "
              "Nnu = Nw - 1 = 2 round(1.5 beta) in {{16,30,60,120}}, lambda_m, all points in one ldga_batch_chain_m call")


def run_batch(args):
    """The uneven (U, beta) scan: every point's chain in flight together (one stream per point)."""
    import torch
    from ladderdga_b200 import _lib
    from ladderdga_b200 import synthetic as S
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pts = S.batch_points(args.points, ns=args.ns or 32)
    main_stream = torch.cuda.current_stream(local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def build(prec):
        chains = [Chain(S.make_input(**p), prec, local, stream=torch.cuda.Stream(local)) for p in pts]
        tuned = {}
        for c in chains:                               # one autotuning run per box size
            if c.ctx.Nnu not in tuned:
                tuned[c.ctx.Nnu] = tune(c)
        scs = [(C.c_double * 8)() for _ in chains]
        ios = {}
        for key, outputs in (("dev", False), ("pin", True)):
            arr = (_lib.ChainIO * len(chains))()
            for i, c in enumerate(chains):
                arr[i] = c.io(c.dev if key == "dev" else c.pin, outputs, scs[i])
            ios[key] = arr
        return chains, tuned, scs, ios

    def timed(chains, ios, key, steps, sel=None):
        """Mean device time of `steps` ldga_batch_chain_m calls over the points `sel` (all: None)."""
        idx = list(range(len(chains))) if sel is None else sel
        sub = [chains[i] for i in idx]
        handles = (C.c_void_p * len(sub))(*[c.ctx.h.value for c in sub])
        arr = (_lib.ChainIO * len(sub))(*[ios[key][i] for i in idx])
        status = (C.c_int32 * len(sub))()
        lib = sub[0].lib
        times = []
        for _ in range(steps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(main_stream)
            for c in sub:
                c.stream.wait_event(a)
            st = lib.ldga_batch_chain_m(len(sub), handles, arr, 1, status)
            if st != 0:
                raise RuntimeError(f"ldga_batch_chain_m failed: {[lib.ldga_last_error(c.ctx.h).decode() for c in sub]}")
            for c in sub:
                e = torch.cuda.Event()
                e.record(c.stream)
                main_stream.wait_event(e)
            b.record(main_stream)
            b.synchronize()
            times.append(a.elapsed_time(b))
        return float(np.mean(times))

    def warm(chains, ios, key):
        handles = (C.c_void_p * len(chains))(*[c.ctx.h.value for c in chains])
        status = (C.c_int32 * len(chains))()
        for _ in range(max(args.warmup, 3)):
            chains[0].lib.ldga_batch_chain_m(len(chains), handles, ios[key], 1, status)
        torch.cuda.synchronize()

    def launches(chains):
        tot = 0
        for c in chains:
            v = C.c_int64()
            c.ctx.call("ldga_launch_count", C.byref(v))
            tot += v.value
        return tot

    chains, tuned, scs, ios = build(PREC_NAMES[args.prec])
    n = len(chains)
    for key in ("dev", "pin"):
        warm(chains, ios, key)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    cnt0 = launches(chains)
    ms = timed(chains, ios, "dev", args.steps)
    cnt1 = launches(chains)
    ms_e2e = timed(chains, ios, "pin", args.steps)
    clk = clocks.stop()
    # each box size's points alone (untimed for the line's value): where the batch's time goes
    few = max(3, args.steps // 4)
    by_box = {}
    for nnu in sorted(tuned):
        sel = [i for i, c in enumerate(chains) if c.ctx.Nnu == nnu]
        by_box[str(nnu)] = {"points": len(sel), "ms": timed(chains, ios, "dev", few, sel)}
    points = sum(c.points for c in chains)
    from ladderdga_b200 import parallel as P
    ms, ms_e2e = P.max_over_ranks(ms), P.max_over_ranks(ms_e2e)
    nnu = sorted({c.ctx.Nnu for c in chains})
    line = {"metric": METRIC, "value": world * points / (ms / 1e3), "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.prec != "mixed" else "f64+f32",
            "data": "synthetic", "impl": "ours", "precision_mode": args.prec,
            "config": {"workload": BATCH_NAME.format(n=n), "global_batch": n * world, "nnu_set": nnu,
                       "bse_config": {str(k): v for k, v in sorted(tuned.items())},
                       "parallelism": f"replicas{world}", "l2": "flushed (256 MiB write) before each step",
                       "points_per_step_per_gpu": points},
            "e2e": {"value": world * points / (ms_e2e / 1e3), "unit": METRIC,
                    "h2d_bytes_per_step": sum(c.h2d_bytes for c in chains),
                    "d2h_bytes_per_step": sum(c.d2h_bytes for c in chains), "ms_per_step": ms_e2e,
                    "path": "C ABI (ldga_batch_chain_m) from pinned host buffers"},
            "gpu_launches": int(cnt1 - cnt0),
            "by_box_size": by_box,
            "by_box_note": "each box size's points alone in one ldga_batch_chain_m call (device time)",
            "clocks": clk}
    if args.prec == "mixed" and not args.no_fp64_compare:
        # the same batch in FP64 mode (LU solves throughout), device-resident inputs
        del chains, ios
        torch.cuda.synchronize()
        c64, tuned64, _, ios64 = build(PREC_NAMES["fp64"])
        warm(c64, ios64, "dev")
        ms64 = P.max_over_ranks(timed(c64, ios64, "dev", few))
        line["fp64_compare"] = {"ms_per_step": ms64, "value": world * points / (ms64 / 1e3), "steps": few,
                                "bse_config": {str(k): v for k, v in sorted(tuned64.items())},
                                "mixed_over_fp64": ms64 / ms}
    if rank == 0:
        print(json.dumps(line), flush=True)
        if args.out:
            open(args.out, "w").write(json.dumps(line) + "\n")
    return 0


def main():
    global TUNE_FILE, BSE_CONFIG
    args = parse()
    TUNE_FILE = args.tune_file
    BSE_CONFIG = (PREC_NAMES[args.prec], args.bse_config) if args.bse_config else None
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.shard == "omega":
        return run_omega_sharded(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
