"""Generate the golden fixtures of the ladder chain (tests/golden/chain_<case>.npz).

LadderDGA.jl's own test suite holds no golden vectors for the ladder chain (its ladderDGATools
testsets are empty and the full run asserts properties only), and Julia is not available to run it,
so the fixtures are the FP64 oracle's outputs (oracle/ldga_ref.py) on seeded synthetic inputs, frozen
here so that the CUDA path and later oracle edits are both checked against the same numbers.  Each
file also stores a digest of its synthetic inputs, so a change of the input generator is detected
instead of silently moving the target.

    python tests/golden/make_golden.py            # rewrite every fixture
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ladderdga_b200 import synthetic as S  # noqa: E402
from oracle import ldga_ref as R  # noqa: E402

HERE = Path(__file__).resolve().parent

# small cases the oracle finishes in well under a second; both lambda corrections converge on each
CASES = {
    "2d8": dict(dim=2, ns=8, beta=5.0, U=1.0, n_iv=4, n_iw=4, seed=81),
    "3d8": dict(dim=3, ns=8, beta=5.0, U=1.2, n_iv=4, n_iw=4, seed=77),
    "2d6_shift": dict(dim=2, ns=6, beta=6.0, U=1.0, n_iv=4, n_iw=3, seed=79, shift=True),
}


def input_digest(inp) -> str:
    h = hashlib.sha256()
    for a in (inp.sigma_loc, inp.gimp, inp.chi_loc_m, inp.chi_loc_d, inp.gamma_m, inp.gamma_d):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(np.array([inp.Ekin_DMFT, inp.Epot_DMFT, inp.sVk, inp.mu, inp.n]).tobytes())
    return h.hexdigest()


def result_arrays(prefix: str, res) -> dict:
    out = {f"{prefix}_scalars": np.array([res.lam_m, res.lam_d, res.mu, res.n, res.EKin, res.EPot_p1, res.EPot_p2,
                                          res.PP_p1, res.PP_p2, float(res.converged)])}
    if res.Sigma_ladder is not None:
        out[f"{prefix}_sigma"] = np.asarray(res.Sigma_ladder)
    return out


def make(name: str) -> dict:
    inp = S.make_input(**CASES[name])
    m = R.run_chain(inp, lambda_type="m")
    dm = R.run_chain(inp, lambda_type="dm")
    h = m["h"]
    data = dict(
        digest=np.array(input_digest(inp)),
        chi0=m["chi0"], chi_m=m["chi_m"].data, chi_d=m["chi_d"].data, gamma_m=m["gamma_m"], gamma_d=m["gamma_d"],
        lambda0=m["lambda0"], gloc=h.G_irr, chiloc_m_sum=np.array(h.chiloc_m_sum), imp_density=np.array(h.imp_density),
    )
    data.update(result_arrays("lm", m["result"]))
    data.update(result_arrays("ldm", dm["result"]))
    return data


def main() -> None:
    for name in CASES:
        np.savez(HERE / f"chain_{name}.npz", **make(name))
        print("wrote", HERE / f"chain_{name}.npz")


if __name__ == "__main__":
    main()
