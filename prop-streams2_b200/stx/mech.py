"""Mechanism and property-table generation for the multi-species reacting step.

The solver consumes the same property tables as the reference: the arrays that
``set_fluid_prop`` / ``set_fluid_prop_cantera`` build in
``src/multideal/multideal.F90:2714-3318`` and that ``tools/preproc_multi/preproc.py``
writes to ``fluid_prop.bin``.  Cantera (the reference's table source, version
3.0.0 per the YAML headers) is not available, so this module restates the parts
of its published algorithms that the tables need:

* species molecular weights from element atomic weights;
* NASA-7 / NASA-9 polynomials for cp, h, s (exact, from the YAML data);
* reaction rate parameters converted to SI kmol units (exact);
* equilibrium constants K_c from the NASA Gibbs energies at p_ref = 1 atm,
  clamped to [tiny, huge] as ``multideal.F90:2918-2923`` does;
* pure-species viscosity, conductivity and binary diffusion coefficients from
  Chapman-Enskog kinetic theory (Neufeld 1972 collision-integral fits, Brokaw
  1969 polar correction, modified Eucken conductivity).  Cantera fits
  polynomials to a more detailed model, so these transport tables are close to,
  but not identical with, the reference's.

All arrays are stored in the reference's Fortran (column-major) order, flattened,
so that they can be handed to the C ABI exactly as the Fortran host would.
"""
from __future__ import annotations

import dataclasses
import math
import re
import struct
from typing import Dict, List, Optional, Sequence

import numpy as np

R_UNIV = 8314.46261815324        # J/(kmol K), src/parameters.F90:53
ONE_ATM = 101325.0
K_BOLTZ = 1.380649e-23
N_AVO = 6.02214076e26            # 1/kmol
DBL_TINY = np.finfo(np.float64).tiny
DBL_HUGE = np.finfo(np.float64).max

# IUPAC atomic weights as used by Cantera 3.0 (kg/kmol)
ATOMIC_WEIGHTS = {
    "H": 1.008, "He": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999,
    "Ar": 39.95, "Ne": 20.1797, "F": 18.998403163, "Cl": 35.45, "S": 32.06,
    "E": 5.485799090649e-4,
}

# reaction type codes used by the kernels (kernels_gpu.F90:9251-9300)
RT_ARRHENIUS, RT_THREEBODY, RT_LINDEMANN, RT_TROE, RT_SRI = 0, 1, 2, 3, 4


@dataclasses.dataclass
class Species:
    name: str
    composition: Dict[str, float]
    mw: float
    nasa_model: str                 # "NASA7" or "NASA9"
    tranges: List[float]            # temperature breakpoints (len = nset + 1)
    coeffs: List[List[float]]       # per range, 7 (NASA7) or 9 (NASA9) coefficients
    geometry: int = 0               # 0 atom, 1 linear, 2 nonlinear
    well_depth: float = 0.0         # epsilon/k [K]
    diameter: float = 0.0           # sigma [Angstrom]
    dipole: float = 0.0             # [Debye]
    polarizability: float = 0.0     # [Angstrom^3]
    rot_relax: float = 0.0


@dataclasses.dataclass
class Reaction:
    equation: str
    reactants: Dict[str, float]
    products: Dict[str, float]
    reversible: bool
    rtype: int
    rate: List[float]               # [A, b, Ea] (SI kmol, J/kmol) or low rate for falloff
    high: Optional[List[float]] = None
    falloff: Optional[List[float]] = None
    efficiencies: Optional[Dict[str, float]] = None
    default_eff: float = 1.0


@dataclasses.dataclass
class Mechanism:
    species: List[Species]
    reactions: List[Reaction]

    @property
    def names(self) -> List[str]:
        return [s.name for s in self.species]

    @property
    def ns(self) -> int:
        return len(self.species)

    @property
    def nr(self) -> int:
        return len(self.reactions)

    def index(self, name: str) -> int:
        low = [n.lower() for n in self.names]
        return low.index(name.lower())


# --------------------------------------------------------------------------- YAML
def _species_mw(comp: Dict[str, float]) -> float:
    mw = 0.0
    for el, n in comp.items():
        key = el if el in ATOMIC_WEIGHTS else el.capitalize()
        mw += ATOMIC_WEIGHTS[key] * float(n)
    return mw


_TERM = re.compile(r"^\s*(\d+(?:\.\d*)?)?\s*(\S+)\s*$")


def _parse_side(side: str):
    """Parse one side of a Cantera equation into ({species: coeff}, collider)."""
    collider = None
    m = re.search(r"\(\+\s*([^)\s]+)\s*\)", side)
    if m:
        collider = ("falloff", m.group(1))
        side = side[:m.start()] + side[m.end():]
    terms = {}
    for tok in side.split(" + "):
        tok = tok.strip()
        if not tok:
            continue
        mt = _TERM.match(tok)
        if mt is None:
            raise ValueError(f"cannot parse term {tok!r}")
        coef = float(mt.group(1)) if mt.group(1) else 1.0
        name = mt.group(2)
        if name == "M":
            collider = ("threebody", "M")
            continue
        terms[name] = terms.get(name, 0.0) + coef
    return terms, collider


def _conv_rate(rc, order: float, units: dict) -> List[float]:
    """Convert a YAML rate constant {A, b, Ea} to SI kmol / J/kmol units."""
    A = float(rc["A"])
    b = float(rc.get("b", 0.0))
    Ea = float(rc.get("Ea", 0.0))
    length = units.get("length", "m")
    quantity = units.get("quantity", "kmol")
    lfac = {"cm": 1e-2, "m": 1.0, "mm": 1e-3}[length]
    qfac = {"mol": 1e-3, "kmol": 1.0, "molec": 1.0 / N_AVO}[quantity]
    # A has units (length^3/quantity)^(order-1) / s
    A *= (lfac ** 3 / qfac) ** (order - 1.0)
    ea_units = units.get("activation-energy", "J/kmol")
    eafac = {"cal/mol": 4184.0, "kcal/mol": 4184000.0, "J/mol": 1000.0,
             "kJ/mol": 1.0e6, "J/kmol": 1.0, "K": R_UNIV}[ea_units]
    return [A, b, Ea * eafac]


def load_yaml_mechanism(path: str) -> Mechanism:
    """Read the subset of Cantera's YAML format the reference examples use."""
    import yaml

    with open(path) as fh:
        doc = yaml.safe_load(fh)
    units = doc.get("units", {})
    phase = doc["phases"][0]
    order = list(phase["species"])
    sp_by_name = {s["name"]: s for s in doc["species"]}
    species = []
    geo_map = {"atom": 0, "linear": 1, "nonlinear": 2}
    for name in order:
        s = sp_by_name[name]
        th = s["thermo"]
        model = th["model"]
        if model == "NASA7":
            tr = [float(t) for t in th["temperature-ranges"]]
            data = [[float(c) for c in d] for d in th["data"]]
            if len(tr) == 2:          # single range: replicate it
                tr = [tr[0], 0.5 * (tr[0] + tr[1]), tr[1]]
                data = [data[0], data[0]]
        elif model == "NASA9":
            tr = [float(t) for t in th["temperature-ranges"]]
            data = [[float(c) for c in d] for d in th["data"]]
        else:
            raise ValueError(f"unsupported thermo model {model}")
        tp = s.get("transport", {})
        species.append(Species(
            name=name, composition=dict(s["composition"]), mw=_species_mw(s["composition"]),
            nasa_model=model, tranges=tr, coeffs=data,
            geometry=geo_map.get(tp.get("geometry", "atom"), 0),
            well_depth=float(tp.get("well-depth", 0.0)), diameter=float(tp.get("diameter", 0.0)),
            dipole=float(tp.get("dipole", 0.0)), polarizability=float(tp.get("polarizability", 0.0)),
            rot_relax=float(tp.get("rotational-relaxation", 0.0))))
    reactions = []
    for r in doc.get("reactions", []):
        eq = r["equation"]
        if "<=>" in eq:
            lhs, rhs = eq.split("<=>")
            rev = True
        elif "=>" in eq:
            lhs, rhs = eq.split("=>")
            rev = False
        else:
            lhs, rhs = eq.split("=")
            rev = True
        reac, col1 = _parse_side(lhs)
        prod, _ = _parse_side(rhs)
        rtype_s = r.get("type", "elementary")
        if "orders" in r:
            raise ValueError("explicit reaction orders are not supported")
        nreac = sum(reac.values())
        eff = None
        deff = 1.0
        if rtype_s == "three-body" or (col1 is not None and col1[0] == "threebody"):
            rtype = RT_THREEBODY
            rate = _conv_rate(r["rate-constant"], nreac + 1.0, units)
            eff = {k: float(v) for k, v in (r.get("efficiencies") or {}).items()}
            deff = float(r.get("default-efficiency", 1.0))
            reactions.append(Reaction(eq, reac, prod, rev, rtype, rate, efficiencies=eff, default_eff=deff))
        elif rtype_s == "falloff":
            low = _conv_rate(r["low-P-rate-constant"], nreac + 1.0, units)
            high = _conv_rate(r["high-P-rate-constant"], nreac, units)
            if col1 is not None and col1[1] != "M":
                eff = {col1[1]: 1.0}
                deff = 0.0
            else:
                eff = {k: float(v) for k, v in (r.get("efficiencies") or {}).items()}
                deff = float(r.get("default-efficiency", 1.0))
            if "Troe" in r:
                t = r["Troe"]
                fo = [float(t["A"]), float(t["T3"]), float(t["T1"])]
                # absent T2 uses the sentinel of cantera_utils_cxx.cxx:228
                fo += [float(t["T2"]) if "T2" in t else -3.14, 0.0]
                rtype = RT_TROE
            elif "SRI" in r:
                t = r["SRI"]
                fo = [float(t["A"]), float(t["B"]), float(t["C"]),
                      float(t.get("D", 1.0)), float(t.get("E", 0.0))]
                rtype = RT_SRI
            else:
                fo = [0.0] * 5
                rtype = RT_LINDEMANN
            reactions.append(Reaction(eq, reac, prod, rev, rtype, low, high=high, falloff=fo,
                                      efficiencies=eff, default_eff=deff))
        elif rtype_s == "elementary":
            rate = _conv_rate(r["rate-constant"], nreac, units)
            reactions.append(Reaction(eq, reac, prod, rev, RT_ARRHENIUS, rate))
        else:
            raise ValueError(f"unsupported reaction type {rtype_s}")
    return Mechanism(species, reactions)


def mechanism_to_dict(mech: Mechanism) -> dict:
    return {"species": [dataclasses.asdict(s) for s in mech.species],
            "reactions": [dataclasses.asdict(r) for r in mech.reactions]}


def mechanism_from_dict(d: dict) -> Mechanism:
    return Mechanism([Species(**s) for s in d["species"]], [Reaction(**r) for r in d["reactions"]])


def restrict_species(mech: Mechanism, keep: Sequence[str], rename: Optional[Dict[str, str]] = None) -> Mechanism:
    """Drop species (and every reaction that involves a dropped species as reactant
    or product); optionally rename species (e.g. an inert Ar -> N2 swap keeps the
    kinetics but takes the new species' thermo/transport from ``rename``'s source)."""
    keep_l = [k.lower() for k in keep]
    sp = [s for s in mech.species if s.name.lower() in keep_l]
    sp.sort(key=lambda s: keep_l.index(s.name.lower()))
    names = {s.name for s in sp}
    rx = []
    for r in mech.reactions:
        if all(k in names for k in r.reactants) and all(k in names for k in r.products):
            r2 = dataclasses.replace(r)
            if r2.efficiencies is not None:
                r2.efficiencies = {k: v for k, v in r2.efficiencies.items() if k in names}
            rx.append(r2)
    return Mechanism(sp, rx)


# --------------------------------------------------------------------------- thermo
def synthetic_mechanism(ns: int = 53, nr: int = 325, seed: int = 0, base: Optional[Species] = None,
                        third_body_frac: float = 0.2) -> Mechanism:
    """The seeded stiff-mechanism workload (no counterpart in the reference,
    which compiles N_S into its kernels, index_define.h): ns species S00.. whose
    NASA-7 coefficients and transport parameters are those of `base` (N2 by
    default) each scaled by U(0.95, 1.05); one molecular weight for all, so that
    every reaction A + B <=> C + D between four distinct random species conserves
    mass; nr reversible reactions with A ~ logU(1e8, 1e16) cm^3/mol/s (cm^6/mol^2/s
    for the third_body_frac of three-body reactions, whose collision efficiencies
    are U(0.5, 5) per species), b ~ U(-1.5, 2), Ea ~ U(0, 50) kcal/mol."""
    rng = np.random.default_rng(seed)
    if base is None:
        base = Species("N2", {"N": 2}, 28.014, "NASA7", [200.0, 1000.0, 5000.0],
                       [[3.298677, 0.0014082404, -3.963222e-06, 5.641515e-09, -2.444854e-12, -1020.8999, 3.950372],
                        [2.92664, 0.0014879768, -5.68476e-07, 1.0097038e-10, -6.753351e-15, -922.7977, 5.980528]],
                       geometry=1, well_depth=97.53, diameter=3.621, polarizability=1.76, rot_relax=4.0)
    species = []
    for k in range(ns):
        f = lambda: float(rng.uniform(0.95, 1.05))
        coeffs = [[c * f() for c in rng_coeffs] for rng_coeffs in base.coeffs]
        species.append(Species(f"S{k:02d}", dict(base.composition), base.mw, "NASA7", list(base.tranges), coeffs,
                               geometry=base.geometry, well_depth=base.well_depth * f(),
                               diameter=base.diameter * f(), dipole=base.dipole,
                               polarizability=base.polarizability * f(), rot_relax=base.rot_relax))
    names = [s.name for s in species]
    reactions = []
    cal = 4.184e6                              # kcal/mol -> J/kmol
    for _ in range(nr):
        a, b, c, d = rng.choice(ns, size=4, replace=False)
        reac = {names[a]: 1.0, names[b]: 1.0}
        prod = {names[c]: 1.0, names[d]: 1.0}
        third = rng.uniform() < third_body_frac
        A = 10.0 ** rng.uniform(8.0, 16.0)
        bexp = float(rng.uniform(-1.5, 2.0))
        Ea = float(rng.uniform(0.0, 50.0)) * cal
        if third:
            A *= (1e-6 / 1e-3) ** 2               # cm^6/mol^2/s -> m^6/kmol^2/s
            eff = {n: float(rng.uniform(0.5, 5.0)) for n in names}
            eq = f"{names[a]} + {names[b]} + M <=> {names[c]} + {names[d]} + M"
            reactions.append(Reaction(eq, reac, prod, True, RT_THREEBODY, [A, bexp, Ea], efficiencies=eff))
        else:
            A *= 1e-6 / 1e-3                       # cm^3/mol/s -> m^3/kmol/s
            eq = f"{names[a]} + {names[b]} <=> {names[c]} + {names[d]}"
            reactions.append(Reaction(eq, reac, prod, True, RT_ARRHENIUS, [A, bexp, Ea]))
    return Mechanism(species, reactions)


def _nasa_eval(sp: Species, T: float):
    """Return (cp/R, h/RT, s/R) for one species at T (range picked like Cantera:
    the low range below the midpoint, the high range at or above it)."""
    tr = sp.tranges
    nset = len(tr) - 1
    r = 0
    for j in range(nset):
        if T >= tr[j]:
            r = j
    r = min(r, nset - 1)
    a = sp.coeffs[r]
    if sp.nasa_model == "NASA7":
        cp = a[0] + a[1] * T + a[2] * T**2 + a[3] * T**3 + a[4] * T**4
        h = a[0] + a[1] * T / 2 + a[2] * T**2 / 3 + a[3] * T**3 / 4 + a[4] * T**4 / 5 + a[5] / T
        s = a[0] * math.log(T) + a[1] * T + a[2] * T**2 / 2 + a[3] * T**3 / 3 + a[4] * T**4 / 4 + a[6]
    else:
        cp = a[0] / T**2 + a[1] / T + a[2] + a[3] * T + a[4] * T**2 + a[5] * T**3 + a[6] * T**4
        h = (-a[0] / T**2 + a[1] * math.log(T) / T + a[2] + a[3] * T / 2 + a[4] * T**2 / 3
             + a[5] * T**3 / 4 + a[6] * T**4 / 5 + a[7] / T)
        s = (-a[0] / T**2 / 2 - a[1] / T + a[2] * math.log(T) + a[3] * T + a[4] * T**2 / 2
             + a[5] * T**3 / 3 + a[6] * T**4 / 4 + a[8])
    return cp, h, s


# --------------------------------------------------------------------------- transport
def _omega22(ts):
    return 1.16145 * ts ** -0.14874 + 0.52487 * np.exp(-0.77320 * ts) + 2.16178 * np.exp(-2.43787 * ts)


def _omega11(ts):
    return (1.06036 * ts ** -0.15610 + 0.19300 * np.exp(-0.47635 * ts)
            + 1.03587 * np.exp(-1.52996 * ts) + 1.76474 * np.exp(-3.89411 * ts))


def _delta_star(sp: Species) -> float:
    if sp.dipole == 0.0 or sp.diameter == 0.0 or sp.well_depth == 0.0:
        return 0.0
    return 1.94e3 * sp.dipole ** 2 / (sp.well_depth * sp.diameter ** 3)


def species_viscosity(sp: Species, T):
    ts = T / sp.well_depth
    om = _omega22(ts) + 0.2 * _delta_star(sp) ** 2 / ts
    m = sp.mw / N_AVO
    sig = sp.diameter * 1e-10
    return (5.0 / 16.0) * np.sqrt(math.pi * m * K_BOLTZ * T) / (math.pi * sig * sig * om)


def species_conductivity(sp: Species, T, mu):
    """Modified Eucken: lambda = mu/W (1.32 Cv + 1.77 R) (molar Cv)."""
    cv = np.array([(_nasa_eval(sp, float(t))[0] - 1.0) * R_UNIV for t in np.atleast_1d(T)])
    return mu / sp.mw * (1.32 * cv + 1.77 * R_UNIV)


def binary_diffusion(sa: Species, sb: Species, T, p):
    """Chapman-Enskog binary diffusion coefficient [m^2/s] at T and p:
    D_ab = 3/16 sqrt(2 pi (k T)^3 / m_ab) / (p pi sigma_ab^2 Omega11*), with
    m_ab the reduced mass of one molecule pair."""
    eps = math.sqrt(sa.well_depth * sb.well_depth)
    sig = 0.5 * (sa.diameter + sb.diameter) * 1e-10
    dstar = math.sqrt(_delta_star(sa) * _delta_star(sb))
    ts = T / eps
    om = _omega11(ts) + 0.19 * dstar ** 2 / ts
    mab = (sa.mw * sb.mw / (sa.mw + sb.mw)) / N_AVO
    return (3.0 / 16.0) * np.sqrt(2.0 * math.pi * K_BOLTZ ** 3 * T ** 3 / mab) / (p * math.pi * sig * sig * om)


# --------------------------------------------------------------------------- tables
@dataclasses.dataclass
class Tables:
    """Property tables in the reference's Fortran layouts (flattened column-major).

    ``cp_coeff``/``cv_coeff`` have shape (ncoef+2, ns, nsetcv) with the first axis
    running over ``indx_cp_l:indx_cp_r+2`` and are already multiplied by R_k, as
    ``multideal.F90:2806-2815`` leaves them."""
    names: List[str]
    ns: int
    nr: int
    mw: np.ndarray
    rgas: np.ndarray
    h298: np.ndarray
    indx_cp_l: int
    indx_cp_r: int
    nsetcv: int
    trange: np.ndarray           # (ns, nsetcv+1)
    cp_coeff: np.ndarray         # (ncp, ns, nsetcv), ncp = indx_cp_r - indx_cp_l + 3
    cv_coeff: np.ndarray
    t_min_tab: float
    t_max_tab: float
    dt_tab: float
    num_t_tab: int
    visc: np.ndarray             # (num_t_tab+1, ns)
    lam: np.ndarray              # (num_t_tab+1, ns)
    diffbin: np.ndarray          # (num_t_tab+1, ns, ns) at pressure p0
    reac_ty: np.ndarray          # (nr,) int32
    is_rev: np.ndarray           # (nr,) int32
    arr_a: np.ndarray            # (nr, 2)
    arr_b: np.ndarray
    arr_ea: np.ndarray
    falloff: np.ndarray          # (nr, 5)
    tb_eff: np.ndarray           # (nr, ns)
    r_coeffs: np.ndarray         # (nr, ns)
    p_coeffs: np.ndarray         # (nr, ns)
    kc_tab: np.ndarray           # (num_t_tab+1, nr)
    sigma: np.ndarray = None
    epsk: np.ndarray = None
    dipole: np.ndarray = None
    polariz: np.ndarray = None
    geometry: np.ndarray = None

    @property
    def ncp(self) -> int:
        return self.indx_cp_r - self.indx_cp_l + 3


def num_t_tab_of(t_min_tab: float, t_max_tab: float, dt_tab: float):
    """``num_t_tab = nint(t_max_tab-t_min_tab)/dt_tab`` then ``dt_tab`` rescaled
    (multideal.F90:3101-3102)."""
    n = int(float(round(t_max_tab - t_min_tab)) / dt_tab)
    return n, (t_max_tab - t_min_tab) / n


def build_tables(mech: Mechanism, p0: float, t_min_tab=200.0, t_max_tab=5500.0, dt_tab=1.0,
                 with_transport=True) -> Tables:
    ns, nr = mech.ns, mech.nr
    model = mech.species[0].nasa_model
    if any(s.nasa_model != model for s in mech.species):
        raise ValueError("mixed NASA models are not supported (preproc.py asserts the same)")
    if model == "NASA7":
        icl, icr, nset = 0, 4, 2
    else:
        icl, icr = -2, 4
        nset = len(mech.species[0].tranges) - 1
    ncp = icr - icl + 3
    mw = np.array([s.mw for s in mech.species])
    rgas = R_UNIV / mw
    trange = np.zeros((ns, nset + 1))
    cp = np.zeros((ncp, ns, nset))
    for k, s in enumerate(mech.species):
        if len(s.tranges) != nset + 1:
            raise ValueError("all species need the same number of temperature ranges")
        trange[k, :] = s.tranges
        for m in range(nset):
            cp[:, k, m] = s.coeffs[m][:ncp]
    cp_r = cp * rgas[None, :, None]
    cv_r = cp_r.copy()
    cv_r[0 - icl, :, :] = cp_r[0 - icl, :, :] - rgas[:, None]
    h298 = np.array([_nasa_eval(s, 298.15)[1] * R_UNIV * 298.15 for s in mech.species])

    ntab, dtt = num_t_tab_of(t_min_tab, t_max_tab, dt_tab)
    T = t_min_tab + np.arange(ntab + 1) * dtt
    visc = np.zeros((ntab + 1, ns))
    lam = np.zeros((ntab + 1, ns))
    diff = np.zeros((ntab + 1, ns, ns))
    if with_transport:
        for k, s in enumerate(mech.species):
            visc[:, k] = species_viscosity(s, T)
            lam[:, k] = species_conductivity(s, T, visc[:, k])
        for a in range(ns):
            for b in range(ns):
                diff[:, a, b] = binary_diffusion(mech.species[a], mech.species[b], T, p0)

    reac_ty = np.zeros(nr, np.int32)
    is_rev = np.zeros(nr, np.int32)
    arr_a = np.zeros((nr, 2)); arr_b = np.zeros((nr, 2)); arr_ea = np.zeros((nr, 2))
    fo = np.zeros((nr, 5)); tb = np.ones((nr, ns)); rc = np.zeros((nr, ns)); pc = np.zeros((nr, ns))
    names_l = [n.lower() for n in mech.names]
    for lr, r in enumerate(mech.reactions):
        reac_ty[lr] = r.rtype
        is_rev[lr] = 1 if r.reversible else 0
        arr_a[lr, 0], arr_b[lr, 0], arr_ea[lr, 0] = r.rate
        if r.high is not None:
            arr_a[lr, 1], arr_b[lr, 1], arr_ea[lr, 1] = r.high
        if r.falloff is not None:
            fo[lr, :] = r.falloff
        if r.efficiencies is not None:
            tb[lr, :] = r.default_eff
            for k, v in r.efficiencies.items():
                if k.lower() in names_l:
                    tb[lr, names_l.index(k.lower())] = v
        for k, v in r.reactants.items():
            rc[lr, names_l.index(k.lower())] += v
        for k, v in r.products.items():
            pc[lr, names_l.index(k.lower())] += v
    kc = np.zeros((ntab + 1, nr))
    if nr:
        g = np.zeros((ntab + 1, ns))     # g/RT
        for k, s in enumerate(mech.species):
            for it, t in enumerate(T):
                _, h, sr = _nasa_eval(s, float(t))
                g[it, k] = h - sr
        dnu = pc - rc                     # (nr, ns)
        dg = g @ dnu.T                    # (ntab+1, nr)
        with np.errstate(over="ignore", under="ignore"):
            kc = np.exp(-dg) * (ONE_ATM / (R_UNIV * T[:, None])) ** dnu.sum(axis=1)[None, :]
        kc = np.where(np.isfinite(kc), kc, DBL_HUGE)
        kc = np.clip(kc, DBL_TINY, DBL_HUGE)
    return Tables(
        names=mech.names, ns=ns, nr=nr, mw=mw, rgas=rgas, h298=h298, indx_cp_l=icl, indx_cp_r=icr,
        nsetcv=nset, trange=trange, cp_coeff=cp_r, cv_coeff=cv_r, t_min_tab=float(t_min_tab),
        t_max_tab=float(t_max_tab), dt_tab=dtt, num_t_tab=ntab, visc=visc, lam=lam, diffbin=diff,
        reac_ty=reac_ty, is_rev=is_rev, arr_a=arr_a, arr_b=arr_b, arr_ea=arr_ea, falloff=fo,
        tb_eff=tb, r_coeffs=rc, p_coeffs=pc, kc_tab=kc,
        sigma=np.array([s.diameter for s in mech.species]),
        epsk=np.array([s.well_depth for s in mech.species]),
        dipole=np.array([s.dipole for s in mech.species]),
        polariz=np.array([s.polarizability for s in mech.species]),
        geometry=np.array([s.geometry for s in mech.species], np.int32))


# --------------------------------------------------------------------------- fluid_prop.bin
def _rec(fh, payload: bytes):
    fh.write(struct.pack("<i", len(payload)))
    fh.write(payload)
    fh.write(struct.pack("<i", len(payload)))


def _f(a, dtype="<f8") -> bytes:
    return np.asarray(a).ravel(order="F").astype(dtype).tobytes()


def write_fluid_prop(path: str, tb: Tables, p0: float):
    """Write the record sequence of ``tools/preproc_multi/preproc.py:202-246``.
    The binary-diffusion record holds values at 1 atm; the reader rescales them
    by 101325/p0 (multideal.F90:2864)."""
    with open(path, "wb") as fh:
        _rec(fh, struct.pack("<ii", tb.ns, tb.nr))
        _rec(fh, b"".join(n.ljust(30).encode()[:30] for n in tb.names))
        _rec(fh, _f(tb.mw)); _rec(fh, _f(tb.rgas)); _rec(fh, _f(tb.h298))
        for arr in (tb.sigma, tb.epsk, tb.dipole, tb.polariz):
            _rec(fh, _f(arr if arr is not None else np.zeros(tb.ns)))
        _rec(fh, _f(tb.geometry if tb.geometry is not None else np.zeros(tb.ns), "<i4"))
        ncoef = 7 if tb.indx_cp_l == 0 else 9
        _rec(fh, struct.pack("<ii", ncoef, tb.nsetcv))
        _rec(fh, _f(tb.trange))
        _rec(fh, _f(tb.cp_coeff / tb.rgas[None, :, None]))
        _rec(fh, _f([tb.t_min_tab, tb.t_max_tab, tb.dt_tab]))
        _rec(fh, _f(tb.visc)); _rec(fh, _f(tb.lam))
        _rec(fh, _f(tb.diffbin * p0 / ONE_ATM))
        if tb.nr > 0:
            _rec(fh, _f(tb.reac_ty, "<i4"))
            for arr in (tb.arr_a, tb.arr_b, tb.arr_ea, tb.falloff, tb.tb_eff, tb.r_coeffs, tb.p_coeffs, tb.kc_tab):
                _rec(fh, _f(arr))


def read_fluid_prop(path: str, p0: float, n_s: int, enable_chemistry: int = 2,
                    arr_preexp_multiplier: float = 1.0) -> Tables:
    """Reader that mirrors ``set_fluid_prop`` (multideal.F90:2763-2926), including
    the cp -> cp*R_k, cv(0) = cp(0) - R_k transformation, the 101325/p0 rescale of
    the diffusion table, the pre-exponential multiplier and the K_c clamp.

    The file carries no reversibility flags; the reference leaves ``isRev``
    unset on this path, and here every reaction is read as reversible."""
    recs = []
    with open(path, "rb") as fh:
        data = fh.read()
    pos = 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        recs.append(data[pos + 4: pos + 4 + n])
        pos += 8 + n
    it = iter(recs)
    ns, nr = struct.unpack("<ii", next(it))
    if ns != n_s:
        raise ValueError("Error! Check number of species in fluid_prop.bin or index_define.h")
    if enable_chemistry > 0 and nr == 0:
        raise ValueError("Error! Chemistry enabled but no reaction provided in yaml")
    raw = next(it)
    names = [raw[30 * k: 30 * k + 30].decode().strip() for k in range(ns)]
    d = lambda: np.frombuffer(next(it), "<f8").copy()
    mw, rgas, h298 = d(), d(), d()
    sigma, epsk, dipole, polariz = d(), d(), d(), d()
    geometry = np.frombuffer(next(it), "<i4").copy()
    ncoef, nset = struct.unpack("<ii", next(it))
    if ncoef == 7:
        icl, icr = 0, 4
    elif ncoef == 9:
        icl, icr = -2, 4
    else:
        raise ValueError("Error! Cp model not supported")
    ncp = icr - icl + 3
    trange = d().reshape((ns, nset + 1), order="F")
    cp = d().reshape((ncp, ns, nset), order="F") * rgas[None, :, None]
    cv = cp.copy()
    cv[0 - icl] = cp[0 - icl] - rgas[:, None]
    tmin, tmax, dtt = d()
    ntab, dtt = num_t_tab_of(tmin, tmax, dtt)
    visc = d().reshape((ntab + 1, ns), order="F")
    lam = d().reshape((ntab + 1, ns), order="F")
    diff = d().reshape((ntab + 1, ns, ns), order="F") * ONE_ATM / p0
    if nr > 0 and enable_chemistry > 0:
        reac_ty = np.frombuffer(next(it), "<i4").copy()
        arr_a = d().reshape((nr, 2), order="F") * arr_preexp_multiplier
        arr_b = d().reshape((nr, 2), order="F")
        arr_ea = d().reshape((nr, 2), order="F")
        fo = d().reshape((nr, 5), order="F")
        tb = d().reshape((nr, ns), order="F")
        rc = d().reshape((nr, ns), order="F")
        pc = d().reshape((nr, ns), order="F")
        kc = np.clip(d().reshape((ntab + 1, nr), order="F"), DBL_TINY, DBL_HUGE)
        is_rev = np.ones(nr, np.int32)
    else:
        nr = 0
        reac_ty = np.zeros(0, np.int32); is_rev = np.zeros(0, np.int32)
        arr_a = arr_b = arr_ea = np.zeros((0, 2)); fo = np.zeros((0, 5))
        tb = rc = pc = np.zeros((0, ns)); kc = np.zeros((ntab + 1, 0))
    return Tables(names=names, ns=ns, nr=nr, mw=mw, rgas=rgas, h298=h298, indx_cp_l=icl, indx_cp_r=icr,
                  nsetcv=nset, trange=trange, cp_coeff=cp, cv_coeff=cv, t_min_tab=float(tmin),
                  t_max_tab=float(tmax), dt_tab=dtt, num_t_tab=ntab, visc=visc, lam=lam, diffbin=diff,
                  reac_ty=reac_ty, is_rev=is_rev, arr_a=arr_a, arr_b=arr_b, arr_ea=arr_ea, falloff=fo,
                  tb_eff=tb, r_coeffs=rc, p_coeffs=pc, kc_tab=kc, sigma=sigma, epsk=epsk, dipole=dipole,
                  polariz=polariz, geometry=geometry)


# --------------------------------------------------------------------------- host thermo helpers
def mixture_cp(tb: Tables, T: float, Y: np.ndarray) -> float:
    """``get_cp`` (multideal.F90:5731-5761): NR locate of the range, then the polynomial."""
    nrange = np.ones(tb.ns, int)
    if tb.nsetcv > 1:
        for k in range(tb.ns):
            jl, ju = 0, tb.nsetcv + 2
            while ju - jl > 1:
                jm = (ju + jl) // 2
                if T >= tb.trange[k, jm - 1]:
                    jl = jm
                else:
                    ju = jm
            nrange[k] = jl
    cp = 0.0
    for l in range(tb.indx_cp_l, tb.indx_cp_r + 1):
        cpl = 0.0
        for k in range(tb.ns):
            m = min(max(nrange[k], 1), tb.nsetcv)
            cpl += tb.cp_coeff[l - tb.indx_cp_l, k, m - 1] * Y[k]
        cp += cpl * T ** l
    return cp


def mixture_e(tb: Tables, T: float, Y: np.ndarray) -> float:
    """``get_e_from_temperature``: sum_k Y_k e_k(T) with e_k from the cv polynomial."""
    return _mixture_poly_int(tb, tb.cv_coeff, T, Y)


def mixture_h(tb: Tables, T: float, Y: np.ndarray) -> float:
    """sum_k Y_k h_k(T) with h_k from the cp polynomial (get_species_h_from_temperature)."""
    return _mixture_poly_int(tb, tb.cp_coeff, T, Y)


def _mixture_poly_int(tb: Tables, coeff: np.ndarray, T: float, Y: np.ndarray) -> float:
    e = 0.0
    for k in range(tb.ns):
        m = 1
        if tb.nsetcv > 1:
            jl, ju = 0, tb.nsetcv + 2
            while ju - jl > 1:
                jm = (ju + jl) // 2
                if T >= tb.trange[k, jm - 1]:
                    jl = jm
                else:
                    ju = jm
            m = min(max(jl, 1), tb.nsetcv)
        c = coeff[:, k, m - 1]
        ek = c[tb.indx_cp_r + 1 - tb.indx_cp_l]
        for l in range(tb.indx_cp_l, tb.indx_cp_r + 1):
            if l == -1:
                ek += c[l - tb.indx_cp_l] * math.log(T)
            else:
                ek += c[l - tb.indx_cp_l] / (l + 1.0) * T ** (l + 1)
        e += ek * Y[k]
    return e


def mixture_viscosity(tb: Tables, T: float, Y: np.ndarray) -> float:
    """``get_mixture_viscosity``: Wilke's rule on the interpolated tables."""
    itt = int((T - tb.t_min_tab) / tb.dt_tab) + 1
    itt = min(max(itt, 1), tb.num_t_tab)
    tl = tb.t_min_tab + (itt - 1) * tb.dt_tab
    f = (T - tl) / tb.dt_tab
    mu_k = tb.visc[itt - 1] + (tb.visc[itt] - tb.visc[itt - 1]) * f
    mu = 0.0
    for l in range(tb.ns):
        den = 0.0
        for m in range(tb.ns):
            phi = 1.0 / math.sqrt(1.0 + tb.mw[l] / tb.mw[m]) * (1.0 + math.sqrt(mu_k[m] / mu_k[l]) * (tb.mw[m] / tb.mw[l]) ** 0.25) ** 2
            den += Y[m] * phi / tb.mw[m]
        mu += mu_k[l] * Y[l] / tb.mw[l] / den
    return math.sqrt(8.0) * mu
