"""Freeze LadderDGA.jl's DMFT test fixture (test/test_data/b1u2_ED_data.jld2, the input of
test/full_run.jl and test/thermodynamics.jl) into files that travel with this repository.

Writes, next to this script:
- ``b1u2_dmft.npz``: every key of the JLD2 file that the plain ladder path and ``calc_E_ED`` read
  (Γsp, Γch, χDMFTsp, χDMFTch, gImp, g0, ϵₖ, Vₖ, U, μ, β, nden, E_kin_DMFT, E_pot_DMFT,
  grid_nBose, grid_nFermi, grid_shift), in Julia's axis order, read by ``ladderdga_b200.jld2``.
  The χ_r asymptotics arrays (only the BSE_SC helpers use them) are left out.
- ``b1u2_plain.toml``: a configuration for that input on the plain path (the reference's
  test/test_data/config_b1u2.toml selects ``chi_asympt_method = "direct"``, which needs BSE_SC.jl;
  here ``"nothing"`` with no ν shell), same lattice (3D simple cubic, t = 1/(2√6), 10³ points).
- ``chain_b1u2.npz``: the FP64 oracle's ladder chain on those inputs (λm correction; the λdm
  Newton does not find a root on this input, which the file records) as compact checks: the full
  χ_m, χ_d and Σ_ladder, scalars, and sums / sampled entries of χ₀, γ_r and λ₀.

    python tests/golden/make_dmft_fixture.py [path/to/b1u2_ED_data.jld2]
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1].parent
sys.path.insert(0, str(ROOT))

from ladderdga_b200 import inputs as I  # noqa: E402
from ladderdga_b200 import jld2  # noqa: E402

HERE = Path(__file__).resolve().parent
# the source file: argument 1, else the fixture inside the LadderDGA.jl checkout named by LDGA_REFERENCE_DIR
DEFAULT_SRC = os.path.join(os.environ.get("LDGA_REFERENCE_DIR", "."), "test", "test_data", "b1u2_ED_data.jld2")
KEYS = ("Γsp", "Γch", "χDMFTsp", "χDMFTch", "gImp", "g0", "ϵₖ", "Vₖ", "U", "μ", "β", "nden",
        "E_kin_DMFT", "E_pot_DMFT", "grid_nBose", "grid_nFermi", "grid_shift")

CONFIG = """# Plain lDΓA path (no χ asymptotics) on LadderDGA.jl's b1u2 DMFT test input.
[Model]
kGrid = "3Dsc-0.2041241452319315"

[Simulation]
Nk = [10]
chi_asympt_method = "nothing"
chi_asympt_shell = 0
usable_prct_reduction = 0.0
omega_smoothing = "nothing"

[Environment]
inputDir = "."
inputVars = "b1u2_dmft.npz"
logfile = "stderr"
loglevel = "debug"

[Debug]
full_EoM_omega = true
"""

# entries of the [Nq, Nν, Nω] arrays kept verbatim (q, ν, ω), 0-based
SAMPLES = [(0, 0, 0), (0, 9, 10), (0, 10, 10), (3, 4, 7), (17, 19, 20), (55, 12, 3), (28, 0, 14)]


def checks(prefix: str, a: np.ndarray) -> dict:
    a = np.asarray(a)
    return {f"{prefix}_sum": np.array(a.sum()), f"{prefix}_abs2": np.array(np.sum(np.abs(a) ** 2)),
            f"{prefix}_samples": np.array([a[s] for s in SAMPLES])}


def chain_fixture(cfg_path: Path) -> dict:
    from oracle import ldga_ref as R
    _, mP, sP, env, kgs = I.readConfig(str(cfg_path))
    inp = I.load_impurity_input(env.inputVars, kgs[0], mP, sP)
    m = R.run_chain(inp, lambda_type="m")
    dm = R.run_chain(inp, lambda_type="dm")
    h, res = m["h"], m["result"]
    out = dict(chi_m=m["chi_m"].data, chi_d=m["chi_d"].data, lm_sigma=np.asarray(res.Sigma_ladder),
               lm_scalars=np.array([res.lam_m, res.lam_d, res.mu, res.n, res.EKin, res.EPot_p1, res.EPot_p2,
                                    res.PP_p1, res.PP_p2, float(res.converged)]),
               chiloc_m_sum=np.array(h.chiloc_m_sum), imp_density=np.array(h.imp_density),
               ldm_root=np.array([dm["result"].lam_m, dm["result"].lam_d]))
    out.update(checks("chi0", m["chi0"]))
    out.update(checks("gamma_m", m["gamma_m"]))
    out.update(checks("gamma_d", m["gamma_d"]))
    out.update(checks("lambda0", m["lambda0"]))
    out["gloc"] = np.asarray(h.G_irr)
    return out


def main() -> None:
    src = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC
    f = jld2.jldopen(src)
    np.savez_compressed(HERE / "b1u2_dmft.npz", **{k: np.asarray(f[k]) for k in KEYS})
    (HERE / "b1u2_plain.toml").write_text(CONFIG)
    np.savez(HERE / "chain_b1u2.npz", **chain_fixture(HERE / "b1u2_plain.toml"))
    for n in ("b1u2_dmft.npz", "b1u2_plain.toml", "chain_b1u2.npz"):
        print("wrote", HERE / n)


if __name__ == "__main__":
    main()
