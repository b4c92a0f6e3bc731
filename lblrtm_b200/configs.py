"""Seeded synthetic inputs for the five benchmark configurations.

There is no line database or atmosphere file here, so every configuration is
generated from a seed with the stated distributions:

* lines: centres uniform in the band, strengths log-uniform, air widths
  uniform 0.04-0.10 cm-1/atm, self width equal to the air width, temperature
  exponents uniform 0.5-0.8, lower-state energies uniform 0-3000 cm-1, no
  pressure shift, ordinary (uncoupled) lines of isotopologue 1;
* atmosphere: level pressures log-spaced 1013.25 -> 0.01 mb, temperature
  288 K falling 6.5 K/km to 11 km, isothermal to 20 km, then +1 K/km,
  altitudes from the hypsometric equation, columns from the pressure
  thickness, and exponential / Gaussian mixing-ratio profiles for H2O, CO2,
  O3 and CH4 (HITRAN molecules 1, 2, 3, 6; masses 18, 44, 48, 16).
"""
import numpy as np

from . import abi

R_DRY = 287.05          # J/(kg K)
G0 = 9.80665            # m/s2
M_AIR = 28.964e-3       # kg/mol
N_A = 6.02214199e23
MOLS = (1, 2, 3, 6)     # H2O, CO2, O3, CH4
NMOL = 7


def gen_lines(n, v1, v2, seed, mols=(1,), s_range=(1e-26, 1e-19), fractions=None):
    """Synthetic TAPE3 records, ascending in wavenumber, 250 per panel."""
    rng = np.random.default_rng(seed)
    if fractions is None:
        fractions = np.full(len(mols), 1.0 / len(mols))
    counts = np.floor(np.asarray(fractions) * n).astype(int)
    counts[0] += n - counts.sum()
    mol = np.concatenate([np.full(c, 100 + m, np.int32) for m, c in zip(mols, counts)])
    vnu = rng.uniform(v1, v2, n)
    lo, hi = np.log10(s_range[0]), np.log10(s_range[1])
    sp = 10.0 ** rng.uniform(lo, hi, n)
    alfa = rng.uniform(0.04, 0.10, n)
    tmpalf = rng.uniform(0.5, 0.8, n)
    epp = rng.uniform(0.0, 3000.0, n)
    mol = rng.permutation(mol)
    order = np.argsort(vnu, kind="stable")
    lines = {
        "vnu": vnu[order].astype(np.float64),
        "sp": sp[order].astype(np.float32),
        "alfa": alfa[order].astype(np.float32),
        "epp": epp[order].astype(np.float32),
        "mol": mol[order].astype(np.int32),
        "hwhms": alfa[order].astype(np.float32),
        "tmpalf": tmpalf[order].astype(np.float32),
        "pshift": np.zeros(n, np.float32),
        "iflg": np.zeros(n, np.int32),
    }
    return lines


def temperature(z_km):
    z = np.asarray(z_km, dtype=np.float64)
    t = np.where(z <= 11.0, 288.0 - 6.5 * z,
                 np.where(z <= 20.0, 288.0 - 6.5 * 11.0, 288.0 - 6.5 * 11.0 + (z - 20.0)))
    return t


def mixing_ratios(z_km):
    z = np.asarray(z_km, dtype=np.float64)
    return {
        1: 1e-2 * np.exp(-z / 2.0),
        2: np.full_like(z, 400e-6),
        3: 8e-6 * np.exp(-((z - 25.0) / 8.0) ** 2),
        6: 1.8e-6 * np.exp(-z / 40.0),
    }


def atmosphere(nlay, psfc=1013.25, ptop=0.01, tpert=None, h2o_scale=1.0):
    """Layer profile (dict of arrays) with nlay layers, surface first."""
    plev = np.logspace(np.log10(psfc), np.log10(ptop), nlay + 1)
    zlev = np.zeros(nlay + 1)
    for i in range(nlay):
        z = zlev[i]
        dz = 0.0
        for _ in range(4):  # hypsometric step with the mid-layer temperature
            tm = temperature(z + 0.5 * dz)
            dz = R_DRY * tm / G0 * np.log(plev[i] / plev[i + 1]) / 1000.0
        zlev[i + 1] = z + dz
    tlev = temperature(zlev)
    zmid = 0.5 * (zlev[:-1] + zlev[1:])
    # layer temperature: mean of the piecewise-linear profile over the layer
    tave = np.array([temperature(np.linspace(zlev[i], zlev[i + 1], 33)).mean()
                     for i in range(nlay)])
    if tpert is not None:
        tave = tave + tpert
        tlev = tlev + np.concatenate([[tpert[0]], 0.5 * (tpert[:-1] + tpert[1:]), [tpert[-1]]])
    pave = 0.5 * (plev[:-1] + plev[1:])
    ncol = (plev[:-1] - plev[1:]) * 100.0 / (G0 * M_AIR / N_A) / 1.0e4
    q = mixing_ratios(zmid)
    q[1] = q[1] * h2o_scale
    wk = np.zeros((nlay, abi.LBL_WKDIM))
    qsum = np.zeros(nlay)
    for m, qm in q.items():
        wk[:, m - 1] = qm * ncol
        qsum += qm
    return {
        "pave": pave, "tave": tave, "pzl": plev[:-1], "pzu": plev[1:],
        "tzl": tlev[:-1], "tzu": tlev[1:], "wk": wk,
        "wbroad": ncol * (1.0 - qsum), "nmol": NMOL, "zlev": zlev,
    }


def mtckd_table(seed, v0=-20.0, dv=10.0, n=2003):
    """Smooth MT_CKD-style H2O continuum table (seeded), netCDF layout."""
    rng = np.random.default_rng(seed)
    v = v0 + dv * np.arange(n)
    a = rng.uniform(0.8, 1.2, 6)
    self_ = (2e-22 * a[0] * np.exp(-np.abs(v) / 280.0)
             + 4e-25 * a[1] * np.exp(-((v - 1600.0) / 350.0) ** 2)
             + 1e-26 * a[2] * np.exp(-((v - 3700.0) / 400.0) ** 2))
    for_ = (6e-24 * a[3] * np.exp(-np.abs(v) / 350.0)
            + 2e-26 * a[4] * np.exp(-((v - 1600.0) / 300.0) ** 2))
    texp = 4.5 * a[5] * np.exp(-np.abs(v) / 3000.0)
    return {"v0": v0, "dv": dv, "self_absco_ref": self_, "for_absco_ref": for_,
            "self_texp": texp, "ref_press": 1013.0, "ref_temp": 296.0}


# ---------------------------------------------------------------------------
# the five configurations
# ---------------------------------------------------------------------------

def config0():
    """One homogeneous H2O layer, 2,000 lines in 600-700 cm-1, OD only."""
    lines = gen_lines(2000, 600.0, 700.0, seed=0, mols=(1,))
    prof = {
        "pave": np.array([1013.25]), "tave": np.array([296.0]),
        "pzl": np.array([1013.25]), "pzu": np.array([1013.25]),
        "tzl": np.array([296.0]), "tzu": np.array([296.0]),
        "wk": np.zeros((1, abi.LBL_WKDIM)), "wbroad": np.array([2.48e24]),
        "nmol": NMOL,
    }
    prof["wk"][0, 0] = 1e22
    run = dict(v1=600.0, v2=700.0, iemit=0, ilblf4=1)
    return {"name": "config0", "lines": lines, "profile": prof, "run": run}


def config1(nlines=50000):
    """60 layers, 4 absorbers, 50,000 lines over 500-1500 cm-1, TOA radiance."""
    lines = gen_lines(nlines, 500.0, 1500.0, seed=1, mols=MOLS)
    prof = atmosphere(60)
    run = dict(v1=500.0, v2=1500.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    return {"name": "config1", "lines": lines, "profile": prof, "run": run}


def config2(nlines=400000, band=(10.0, 3000.0), sample=4.0):
    """Precision sweep: 400,000 lines over 10-3000 cm-1 plus a continuum."""
    lines = gen_lines(nlines, band[0], band[1], seed=2, mols=MOLS,
                      s_range=(1e-28, 1e-18))
    prof = atmosphere(60)
    run = dict(iemit=1, ilblf4=1, icntnm=1, tmpbnd=290.0, bndemi=0.98,
               sample=sample)
    # reference-legal sub-runs (V2-V1 <= 2020 cm-1)
    subruns = [(10.0, 1505.0), (1505.0, 3000.0)]
    return {"name": "config2", "lines": lines, "profile": prof, "run": run,
            "subruns": subruns, "mtckd": mtckd_table(2)}


def config3(nlines=200000):
    """Jacobians: config-1 profile over 650-2500 cm-1, 200,000 lines."""
    lines = gen_lines(nlines, 650.0, 2500.0, seed=3, mols=MOLS)
    prof = atmosphere(60)
    run = dict(v1=650.0, v2=2500.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    return {"name": "config3", "lines": lines, "profile": prof, "run": run,
            "jac_mols": (1, 3)}


def config4(nprof=256, nlines=200000, seed=4):
    """256 perturbed profiles with 30-90 layers, 200,000 lines 600-2500 cm-1."""
    rng = np.random.default_rng(seed)
    lines = gen_lines(nlines, 600.0, 2500.0, seed=seed, mols=MOLS)
    profs = []
    for _ in range(nprof):
        nl = int(rng.integers(30, 91))
        noise = rng.normal(0.0, 5.0, nl)
        sm = np.convolve(np.pad(noise, 1, mode="edge"), np.ones(3) / 3.0, mode="valid")
        scale = float(np.exp(rng.normal(0.0, 0.3)))
        profs.append(atmosphere(nl, tpert=sm, h2o_scale=scale))
    run = dict(v1=600.0, v2=2500.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    return {"name": "config4", "lines": lines, "profiles": profs, "run": run,
            "jac_mols": (1, 3)}


def subset_lines(lines, v1, v2, margin=25.0):
    """Lines within [v1-margin, v2+margin] (a sub-run's TAPE3 extract)."""
    m = (lines["vnu"] >= v1 - margin) & (lines["vnu"] <= v2 + margin)
    return {k: v[m] for k, v in lines.items()}
