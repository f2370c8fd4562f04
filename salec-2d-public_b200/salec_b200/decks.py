"""Seeded synthetic input decks and EOS files in the reference's own formats.

The reference ships no EOS tables (its eos/ folder holds only eos-help.txt), so every deck
used by the tests and the benchmark is generated here:

* ``.inp`` decks in the ``[section] key = value`` format read by the reference's
  ``OpenInputFile`` (src/io/InputParser.c:225-281) and interpreted by ``load_mesh_info``
  (src/sale2d_back.c:64-247), ``load_state_reference`` (:250-402), ``load_target_info``
  (src/target_profile.c:345-484) and ``load_projectile_info`` (src/sale2d_back.c:29-62).
  Per-material keys are always written as lists, because ``GetValueDk`` reads an
  uninitialised buffer for a non-list value (src/io/InputParser.c:433-449).
* Tillotson key files (``<name>.tillotson``) with the keys of ``LoadTillEOS``
  (src/eos/eos_state.c:635-662).
* ANEOS "SieDen" tables (``<name>.aneos.sd``) in the layout of ``LoadANEOSSieDen``
  (src/eos/aneos_sieden.c:11-73): three comment lines, ``nDen nTem``, ``Pnorm Tnorm``,
  nTem specific-energy nodes, nDen density nodes, nDen x nTem triples (T, p, c) with the
  energy index fastest, then nDen x nTem (entropy, strength) pairs that the reader skips.

Materials are generic Tillotson parameter sets; the tabulated granite is generated from the
Tillotson formulas (restated in ``tillotson_pc``) on a seeded grid.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional

import numpy as np

# name -> Tillotson constants (SI units). Cv is the specific heat used for temperature.
TILLOTSON = {
    "basalt_": dict(Rho0=2700.0, BulkA=2.67e10, BulkB=2.67e10, E0=4.87e8, Ta=0.5, Tb=1.5,
                    Alpha=5.0, Beta=5.0, Eiv=4.72e6, Ecv=1.82e7, Cv=840.0),
    "granit_": dict(Rho0=2680.0, BulkA=1.80e10, BulkB=1.80e10, E0=1.60e7, Ta=0.5, Tb=1.3,
                    Alpha=5.0, Beta=5.0, Eiv=3.50e6, Ecv=1.80e7, Cv=790.0),
    "ice____": dict(Rho0=917.0, BulkA=9.99e9, BulkB=6.50e9, E0=1.00e7, Ta=0.3, Tb=0.1,
                    Alpha=10.0, Beta=5.0, Eiv=7.73e5, Ecv=3.04e6, Cv=2050.0),
    "dunite_": dict(Rho0=3320.0, BulkA=1.31e11, BulkB=4.90e10, E0=5.50e8, Ta=0.5, Tb=1.5,
                    Alpha=5.0, Beta=5.0, Eiv=4.50e6, Ecv=1.45e7, Cv=1000.0),
    "regolit": dict(Rho0=2700.0, BulkA=2.67e10, BulkB=2.67e10, E0=4.87e8, Ta=0.5, Tb=1.5,
                    Alpha=5.0, Beta=5.0, Eiv=4.72e6, Ecv=1.82e7, Cv=840.0),
}


@dataclasses.dataclass
class Material:
    name: str
    eos: str = "tillotson"          # "tillotson" or "aneos.sd"
    poisson: float = 0.25
    yshear: str = "RockStrengthT"
    yint0: float = 1.0e7
    yintfri: float = 1.2
    yintlim: float = 2.5e9
    ydam0: float = 1.0e7
    ydamfri: float = 1.2
    ydamlim: float = 2.5e9
    damage: str = "Ivanov"
    ytens: str = "SimpleTensile"
    yten0: float = 1.0e7
    simon_a: float = 6.0e9
    simon_c: float = 3.0
    simon_t0: float = 1373.0
    ohnaka_xi: float = 1.2
    toff: float = -1.0              # ACFL switched off unless > 0
    cvib: float = 0.1
    vibmax: float = 200.0
    block_size: float = -1.0
    gamma_eta: float = 8.0e-3
    gamma_beta: float = 115.0
    porosity: str = "None"
    alpha0: float = 1.0
    alphax: float = 1.0
    epse0: float = -1.0e-5
    kappa: float = 0.98
    chi: float = 1.0
    # Johnson-Cook keys (material.JcA ... material.JCMaxPlastic, src/sale2d_back.c:299-306); the
    # deck carries them only when some material sets them, with the reference's defaults for
    # the others
    jc: Optional[Dict[str, float]] = None
    # material.Tdelta, the shift of the melting temperature in the Ohnaka softening
    # (src/sale2d_back.c:339); written only when some material sets it
    tdelta: float = 0.0


# defaults of the Johnson-Cook keys in load_state_reference (src/sale2d_back.c:299-306)
JC_DEFAULTS = {"JcA": 4.90e7, "JcB": 1.57e8, "JcN": 1.67e-1, "JcC": 1.60e-2, "JcM": 1.70, "JcTref": 8.00e2,
               "JcminP": -2.44e9, "JCMaxPlastic": 10.0}


@dataclasses.dataclass
class Deck:
    """One synthetic impact: a layered plane target hit by a spherical projectile."""
    npx: int = 32
    npy: int = 48
    dx: float = 50.0
    dy: float = 50.0
    oy: float = 0.6
    materials: List[Material] = dataclasses.field(default_factory=lambda: [Material("basalt_")])
    target_materials: List[str] = dataclasses.field(default_factory=lambda: ["basalt_"])
    target_depths: List[float] = dataclasses.field(default_factory=lambda: [1.0e6])
    max_depth: float = 0.0          # 0 -> 2 * domain depth
    projectile: str = "basalt_"
    radius_cells: float = 6.0
    velocity: float = -6000.0
    vx: float = 0.0
    gravity: float = -1.62
    damping: str = "pml"
    damp_x: int = 6
    damp_y: int = 6
    lambda_x: float = 10.0
    lambda_y: float = 10.0
    maxstep: int = 20
    dt0: float = 1.0e-3
    maxdt: float = 0.05
    time1: float = 1.0e4
    left: str = "freeslip"
    right: str = "freeslip"
    bottom: str = "fixed"
    top: str = "outflow"
    anc: float = 0.1
    ancpat: str = "pml"
    avisq: float = 1.2
    avisl: float = 0.5
    min_density: float = 1.0e-2
    max_velocity: float = -1.63
    tensile_failure: int = 0
    tracer_strip: int = 2
    temperature: str = "const"
    surf_dtdz: float = 0.0
    ejecta_threshold: float = 2.0
    # ejecta drag (src/ejecta.c:65-133): the reference's defaults are resistance -1, friction 0
    ejecta_resistance: float = -1.0
    ejecta_friction: float = 0.0
    target_temperature: float = 293.0
    projectile_temperature: float = 293.0
    projectile_pressure: float = 1.0e-5
    # write every number with 17 significant digits (the exact double), e.g. for finite
    # differences of a material parameter; False keeps the 6-digit form
    exact: bool = False
    extra: Dict[str, Dict[str, str]] = dataclasses.field(default_factory=dict)


def _lst(values) -> str:
    return "[" + ", ".join(values) + "]"


def _mat_list(mats: List[Material], attr: str, fmt=lambda v: repr(v)) -> str:
    return _lst([""] + [fmt(getattr(m, attr)) for m in mats])


def _g(v: float) -> str:
    return "%.6g" % v


def write_tillotson(path: str, name: str, rho_step: int = 1501) -> None:
    p = TILLOTSON[name]
    with open(path, "w") as f:
        f.write("# Tillotson constants for %s (synthetic parameter set)\n" % name)
        f.write("[Tillostson]\n")
        for k in ("Rho0", "BulkA", "BulkB", "E0", "Ta", "Tb", "Alpha", "Beta", "Eiv", "Ecv"):
            f.write("    %s = %.10g\n" % (k, p[k]))
        f.write("[ColdEnergy]\n")
        f.write("    Cv = %.10g\n" % p["Cv"])
        f.write("    Tref = 293.0\n")
        f.write("    RhoStep = %d\n" % rho_step)


def tillotson_pc(p: dict, eng: np.ndarray, rho: np.ndarray):
    """Tillotson pressure and sound speed (cold, hot and transition branches).

    Restates the published Tillotson (1962) equation of state as evaluated by the reference's
    TillCold/TillHot/TillTran/TillPres (src/eos/eos_state.c:322-438), vectorised with numpy.
    Used only to generate synthetic tables.
    """
    rho0, A, B, E0 = p["Rho0"], p["BulkA"], p["BulkB"], p["E0"]
    a, b, al, be, Eiv, Ecv = p["Ta"], p["Tb"], p["Alpha"], p["Beta"], p["Eiv"], p["Ecv"]
    eta = rho / rho0
    mu = eta - 1.0
    phi1 = 1.0 / (eng / (E0 * eta * eta) + 1.0)
    bb = np.where(eta < 1.0, A, B)
    pc = (a + b * phi1) * eng * rho + A * mu + bb * mu * mu
    cc1 = (A + 2 * bb * mu) / rho0 + eng * (a + b * phi1 * (3 - 2 * phi1))
    cc2 = (a + b * phi1 * phi1) * pc / rho
    xi = rho0 / rho - 1.0
    ea = np.where(al * xi * xi < 100.0, np.exp(-np.minimum(al * xi * xi, 100.0)), 0.0)
    eb = np.where(be * xi < 100.0, np.exp(-np.minimum(be * xi, 100.0)), 0.0)
    ph = a * rho * eng + (b * eng * rho * phi1 + A * mu * eb) * ea
    ch1 = (a * eng + b * eng * phi1 * (3 + 2 * al * xi / eta - 2 * phi1) * ea
           + A / rho0 * (1 - (xi / eta) * (be + 2 * al * xi)) * ea * eb)
    ch2 = (a + b * phi1 * phi1 * ea) * ph / rho
    cold = (rho >= rho0) | (eng < Eiv)
    hot = (~cold) & (eng > Ecv)
    dEr, dEl, dT = eng - Eiv, Ecv - eng, Ecv - Eiv
    pt = (dEl * pc + dEr * ph) / dT
    c2c_t = cc1 + (a + b * phi1 * phi1) * pt / rho
    c2h_t = ch1 + (a + b * phi1 * phi1 * ea) * pt / rho
    ct2 = (dEl * c2c_t + dEr * c2h_t) / dT + (ph - pc) / dT * pt / (rho * rho)
    pres = np.where(cold, pc, np.where(hot, ph, pt))
    c2 = np.where(cold, cc1 + cc2, np.where(hot, ch1 + ch2, ct2))
    cs = np.where(c2 < 1e-2, -np.sqrt(np.abs(c2)), np.sqrt(np.abs(c2)))
    cs = np.where(pres <= 1e-2, math.sqrt(A / rho0), cs)
    return pres, cs


def cold_energy(p: dict, rho: np.ndarray, n: int = 4001) -> np.ndarray:
    """Specific energy along the zero-temperature isentrope dE/drho = p/rho^2 through (rho0, 0).

    Fourth-order Runge-Kutta on a uniform density grid, then linear interpolation to ``rho``.
    """
    rho0 = p["Rho0"]
    grid_hi = np.linspace(rho0, max(rho0 * 10.0, float(rho.max()) * 1.01), n)
    grid_lo = np.linspace(rho0, max(float(rho.min()) * 0.99, 1e-3 * rho0), n)

    def integrate(grid):
        e = np.zeros_like(grid)
        for k in range(1, len(grid)):
            h = grid[k] - grid[k - 1]
            r0 = grid[k - 1]
            f = lambda ee, rr: tillotson_pc(p, np.array([ee]), np.array([rr]))[0][0] / (rr * rr)
            k1 = f(e[k - 1], r0)
            k2 = f(e[k - 1] + 0.5 * h * k1, r0 + 0.5 * h)
            k3 = f(e[k - 1] + 0.5 * h * k2, r0 + 0.5 * h)
            k4 = f(e[k - 1] + h * k3, r0 + h)
            e[k] = e[k - 1] + h * (k1 + 2 * k2 + 2 * k3 + k4) / 6.0
        return e

    e_hi, e_lo = integrate(grid_hi), integrate(grid_lo)
    x = np.concatenate([grid_lo[::-1], grid_hi[1:]])
    y = np.concatenate([e_lo[::-1], e_hi[1:]])
    return np.interp(rho, x, y)


def write_sieden(path: str, name: str, nden: int = 512, neng: int = 512, seed: int = 7) -> None:
    """Tabulated (density x specific energy) -> (T, p, c) table generated from Tillotson.

    Density nodes span [0.05, 4] rho0 and energy nodes [0, 4e8] J/kg, both geometrically
    stretched with seeded jitter of the interior nodes (sorted, so strictly increasing);
    T = (E - E_cold(rho)) / Cv + 293 K, clipped at 1 K.
    """
    p = TILLOTSON[name]
    rng = np.random.default_rng(seed)
    rho0 = p["Rho0"]
    u = np.linspace(0.0, 1.0, nden)
    yden = 0.05 * rho0 * (80.0 ** u)
    yden[1:-1] *= 1.0 + 0.2 * (rng.random(nden - 2) - 0.5) / nden
    yden = np.sort(yden)
    v = np.linspace(0.0, 1.0, neng)
    xeng = 4.0e8 * (np.expm1(6.0 * v) / np.expm1(6.0))
    xeng[1:-1] *= 1.0 + 0.2 * (rng.random(neng - 2) - 0.5) / neng
    xeng = np.sort(xeng)
    ec = cold_energy(p, yden)
    E, R = np.meshgrid(xeng, yden)          # [den][eng]
    pres, cs = tillotson_pc(p, E, R)
    tem = np.maximum((E - ec[:, None]) / p["Cv"] + 293.0, 1.0)
    with open(path, "w") as f:
        f.write("# synthetic SieDen table for %s, generated from Tillotson constants\n" % name)
        f.write("# seed %d, %d densities x %d specific energies\n" % (seed, nden, neng))
        f.write("# columns: temperature pressure soundspeed\n")
        f.write("%d %d\n" % (nden, neng))
        f.write("%.15e %.15e\n" % (1.0e5, 293.0))
        f.write("\n".join("%.15e" % x for x in xeng) + "\n")
        f.write("\n".join("%.15e" % y for y in yden) + "\n")
        for j in range(nden):
            rows = np.stack([tem[j], pres[j], cs[j]], axis=1)
            f.write("\n".join("%.15e %.15e %.15e" % tuple(r) for r in rows) + "\n")
        zeros = "\n".join("0.0 0.0" for _ in range(neng)) + "\n"
        for j in range(nden):
            f.write(zeros)


def write_aneos_td(path: str, name: str, ntem: int = 120, nden: int = 160, seed: int = 11) -> None:
    """Tabulated (temperature x density) -> (specific energy, p, c) table in the layout of
    LoadANEOS (src/eos/eos_state.c:89-146), generated from Tillotson constants.

    Layout: three comment lines, ``nTem nDen``, ``Tnorm Dnorm Pnorm``, nTem temperature nodes,
    nTem x nDen triples (E, p, c) with the density index fastest, then nDen density nodes (the
    reader multiplies E by the density). Temperatures span [150 K, 1.5e5 K] and densities
    [0.05, 4] rho0, both geometrically stretched with seeded jitter of the interior nodes
    (sorted, so strictly increasing); E = E_cold(rho) + Cv (T - 293 K), which increases with T
    at every density, as the reader's energy bisection needs.
    """
    p = TILLOTSON[name]
    rng = np.random.default_rng(seed)
    rho0 = p["Rho0"]
    u = np.linspace(0.0, 1.0, ntem)
    xtem = 150.0 * (1000.0 ** u)
    xtem[1:-1] *= 1.0 + 0.2 * (rng.random(ntem - 2) - 0.5) / ntem
    xtem = np.sort(xtem)
    v = np.linspace(0.0, 1.0, nden)
    yden = 0.05 * rho0 * (80.0 ** v)
    yden[1:-1] *= 1.0 + 0.2 * (rng.random(nden - 2) - 0.5) / nden
    yden = np.sort(yden)
    ec = cold_energy(p, yden)
    T, R = np.meshgrid(xtem, yden, indexing="ij")          # [tem][den]
    E = ec[None, :] + p["Cv"] * (T - 293.0)
    pres, cs = tillotson_pc(p, E, R)
    with open(path, "w") as f:
        f.write("# synthetic ANEOS temperature-density table for %s, generated from Tillotson constants\n" % name)
        f.write("# seed %d, %d temperatures x %d densities\n" % (seed, ntem, nden))
        f.write("# columns: specific energy, pressure, sound speed\n")
        f.write("%d %d\n" % (ntem, nden))
        f.write("%.15e %.15e %.15e\n" % (293.0, rho0, 1.0e5))
        f.write("\n".join("%.15e" % x for x in xtem) + "\n")
        for i in range(ntem):
            rows = np.stack([E[i], pres[i], cs[i]], axis=1)
            f.write("\n".join("%.15e %.15e %.15e" % tuple(r) for r in rows) + "\n")
        f.write("\n".join("%.15e" % y for y in yden) + "\n")


def write_deck(deck: Deck, folder: str, stem: str = "deck") -> str:
    """Write ``folder/<stem>.inp`` plus one EOS file per material; return the deck path."""
    os.makedirs(folder, exist_ok=True)
    mats = deck.materials
    for m in mats:
        if m.eos == "tillotson":
            write_tillotson(os.path.join(folder, m.name + ".tillotson"), m.name)
        elif m.eos == "aneos.sd":
            fn = os.path.join(folder, m.name + ".aneos.sd")
            if not os.path.exists(fn):
                write_sieden(fn, m.name)
        elif m.eos in ("aneos", "aneos.td"):
            fn = os.path.join(folder, m.name + "." + m.eos)
            if not os.path.exists(fn):
                write_aneos_td(fn, m.name)
        else:
            raise ValueError("unsupported eos " + m.eos)
    _g = (lambda v: "%.17g" % v) if deck.exact else globals()["_g"]
    radius = deck.radius_cells * deck.dy
    depth_total = deck.npy * deck.oy * deck.dy
    max_depth = deck.max_depth if deck.max_depth > 0 else 2.0 * depth_total
    lines = []
    w = lines.append
    w("# synthetic deck written by salec_b200.decks")
    w("[processor]")
    w("    npgx = 1")
    w("    npgy = 1")
    w("[mesh]")
    w("    dx = %s" % _g(deck.dx))
    w("    dy = %s" % _g(deck.dy))
    w("    npx = %d" % deck.npx)
    w("    npy = %d" % deck.npy)
    w("    Oy = %s" % _g(deck.oy))
    w("    Ox = 0.0")
    w("    ext = off")
    w("[cycle]")
    w("    dt0 = %s" % _g(deck.dt0))
    w("    maxdt = %s" % _g(deck.maxdt))
    w("    time0 = 0.0")
    w("    time1 = %s" % _g(deck.time1))
    w("    maxstep = %d" % deck.maxstep)
    w("[output]")
    w("    prefix = Synth")
    w("    format = binary")
    w("    time = 1.0e9")
    w("    init = 0")
    w("    out_cycle = -1")
    w("[projectile]")
    w("    material = %s" % deck.projectile)
    w("    radiu = %s" % _g(radius))
    w("    center = [%s, %s]" % (_g(0.0), _g(radius)))
    w("    velocity = [%s, %s]" % (_g(deck.vx), _g(deck.velocity)))
    w("    damage = [const, 0.0]")
    w("    pressure = [const, %s]" % ("1.0e-5" if deck.projectile_pressure == 1.0e-5 else _g(deck.projectile_pressure)))
    w("    temperature = [const, %s]" % _g(deck.projectile_temperature))
    w("[target]")
    w("    type = plane")
    w("    number = %d" % len(deck.target_materials))
    w("    material = %s" % _lst(deck.target_materials))
    w("    depth = %s" % _lst([_g(d) for d in deck.target_depths]))
    w("    max_depth = %s" % _g(max_depth))
    if deck.temperature == "const":
        w("    temperature = [const, %s]" % _g(deck.target_temperature))
    else:
        w("    temperature = [conductive, %s]" % _g(deck.target_temperature))
        w("    surf_dtdz = %s" % _g(deck.surf_dtdz))
        w("    r_planet = 1.74e6")
    w("[condition]")
    w("    gravity = [0.0, %s]" % _g(deck.gravity))
    w("[boundary]")
    w("    bottom = %s" % deck.bottom)
    w("    top = %s" % deck.top)
    w("    left = %s" % deck.left)
    w("    right = %s" % deck.right)
    w("[material]")
    w("    nm = %d" % (len(mats) + 1))
    w("    postfix = %s" % _lst(["null"] + [m.eos for m in mats]))
    w("    name = %s" % _lst(["vacuum_"] + [m.name for m in mats]))
    f = lambda attr: _mat_list(mats, attr, _g)
    s = lambda attr: _mat_list(mats, attr, str)
    w("    Poisson = %s" % f("poisson"))
    w("    SimonA = %s" % f("simon_a"))
    w("    SimonC = %s" % f("simon_c"))
    w("    SimonT0 = %s" % f("simon_t0"))
    w("    OhnakaXi = %s" % f("ohnaka_xi"))
    w("    yshear = %s" % s("yshear"))
    w("    yint0 = %s" % f("yint0"))
    w("    yintfri = %s" % f("yintfri"))
    w("    yintlim = %s" % f("yintlim"))
    w("    ydam0 = %s" % f("ydam0"))
    w("    ydamfri = %s" % f("ydamfri"))
    w("    ydamlim = %s" % f("ydamlim"))
    w("    ytens = %s" % s("ytens"))
    w("    yten0 = %s" % f("yten0"))
    w("    damage = %s" % s("damage"))
    w("    BlockSize = %s" % f("block_size"))
    w("    GammaEta = %s" % f("gamma_eta"))
    w("    GammaBeta = %s" % f("gamma_beta"))
    w("    Toff = %s" % f("toff"))
    w("    Cvib = %s" % f("cvib"))
    w("    VibMax = %s" % f("vibmax"))
    w("    Porosity = %s" % s("porosity"))
    w("    alpha0 = %s" % f("alpha0"))
    w("    alphax = %s" % f("alphax"))
    w("    epse0 = %s" % f("epse0"))
    w("    kappa = %s" % f("kappa"))
    w("    chi = %s" % f("chi"))
    if any(m.tdelta != 0.0 for m in mats):
        w("    Tdelta = %s" % f("tdelta"))
    if any(m.jc for m in mats):
        for key, dflt in JC_DEFAULTS.items():
            w("    %s = %s" % (key, _lst([""] + [_g((m.jc or {}).get(key, dflt)) for m in mats])))
    w("[ejecta]")
    w("    threshold = %s" % _g(deck.ejecta_threshold))
    if deck.ejecta_resistance != -1.0:
        w("    resistance = %s" % _g(deck.ejecta_resistance))
    w("    friction = %s" % ("0.0" if deck.ejecta_friction == 0.0 else _g(deck.ejecta_friction)))
    w("[numerical]")
    w("    AVISQ = %s" % _g(deck.avisq))
    w("    AVISL = %s" % _g(deck.avisl))
    w("    ANC = %s" % _g(deck.anc))
    w("    ANCPAT = %s" % deck.ancpat)
    w("    MaxVelocity = %s" % _g(deck.max_velocity))
    w("    MinDensity = %s" % _g(deck.min_density))
    w("    damping = %s" % deck.damping)
    w("    DampX = %d" % deck.damp_x)
    w("    DampY = %d" % deck.damp_y)
    w("    LambdaX = %s" % _g(deck.lambda_x))
    w("    LambdaY = %s" % _g(deck.lambda_y))
    w("    partpres = 0")
    w("    tensile_failure = %d" % deck.tensile_failure)
    w("    tarcer_strip = %d" % deck.tracer_strip)
    for sec, kv in deck.extra.items():
        w("[%s]" % sec)
        for k, v in kv.items():
            w("    %s = %s" % (k, v))
    for ln in lines:
        if "=" in ln and len(ln.split("=", 1)[1].strip()) >= 100:
            raise ValueError("deck value longer than the reference parser's 100 chars: " + ln)
    path = os.path.join(folder, stem + ".inp")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path


def config1_deck(maxstep: int = 999) -> Deck:
    """200 x 400 cells at 50 m, basalt Tillotson target and projectile (20 cells, 6 km/s),
    cohesion 10 MPa, friction 1.2, limit 2.5 GPa, gravity 1.62, 30-layer PML, 1000 steps."""
    return Deck(npx=200, npy=400, dx=50.0, dy=50.0, oy=0.6,
                materials=[Material("basalt_")], target_materials=["basalt_"],
                target_depths=[1.0e6], projectile="basalt_", radius_cells=20.0,
                velocity=-6000.0, gravity=-1.62, damping="pml", damp_x=30, damp_y=30,
                maxstep=maxstep, dt0=1.0e-3, maxdt=0.05)


def config2_deck(n: int = 2048, maxstep: int = 4999) -> Deck:
    """n x n cells, granite target on a tabulated (SieDen) EOS, ice projectile at CPPR 40 and
    15 km/s, rock strength with scalar damage, 30-layer PML."""
    granite = Material("granit_", eos="aneos.sd", poisson=0.25)
    ice = Material("ice____", eos="tillotson", poisson=0.33, yint0=1.0e6, yintfri=0.8,
                   yintlim=1.0e9, ydam0=1.0e4, ydamfri=0.6, ydamlim=1.0e9, simon_t0=273.0)
    return Deck(npx=n, npy=n, dx=50.0, dy=50.0, oy=0.5,
                materials=[granite, ice], target_materials=["granit_"], target_depths=[1.0e7],
                projectile="ice____", radius_cells=40.0, velocity=-15000.0, gravity=-1.62,
                damping="pml", damp_x=30, damp_y=30, maxstep=maxstep, dt0=1.0e-4, maxdt=0.05)


def config3_deck(n: int = 4096, maxstep: int = 2999, dx: float = 50.0, regolith: float = 500.0,
                 basalt: float = 3000.0, cppr: float = 30.0, side_layers: int = 50, base_layers: int = 30) -> Deck:
    """Layered three-material target, n x n cells: porous regolith (25% porosity, Wunnemann
    compaction, cohesion 0.1 MPa) over basalt over a dunite half-space (Tillotson rho0 3320),
    basalt projectile at CPPR 30 and 10 km/s. The reference has one damping type for the whole
    mesh; its PML takes the side and base layer counts separately (DampX 50, DampY 30). The
    seeded density noise of the configuration is applied to the initialised state by
    density_noise()."""
    regol = Material("regolit", poisson=0.25, yint0=1.0e5, yintfri=0.6, yintlim=1.0e9, ydam0=1.0e3,
                     ydamfri=0.4, ydamlim=1.0e9, porosity="Wunnemann", alpha0=1.0 / 0.75, alphax=1.1,
                     epse0=-1.0e-5, kappa=0.98, chi=0.5)
    bas = Material("basalt_")
    dun = Material("dunite_", poisson=0.28)
    return Deck(npx=n, npy=n, dx=dx, dy=dx, oy=0.5, materials=[regol, bas, dun],
                target_materials=["regolit", "basalt_", "dunite_"], target_depths=[regolith, basalt, 1.0e7],
                projectile="basalt_", radius_cells=cppr, velocity=-10000.0, gravity=-1.62, damping="pml",
                damp_x=side_layers, damp_y=base_layers, maxstep=maxstep, dt0=1.0e-4, maxdt=0.05)


def density_noise(m_den: np.ndarray, e_den: np.ndarray, seed: int = 3, amplitude: float = 0.01):
    """Seeded cell-by-cell noise of +-amplitude on the initial density field: every material
    density of a cell and the cell density are scaled by the same factor 1 + amplitude * U(-1, 1),
    drawn once per cell (the noise's correlation length is the cell size). Returns new arrays."""
    rng = np.random.default_rng(seed)
    f = 1.0 + amplitude * (2.0 * rng.random(e_den.shape[:2]) - 1.0)
    md = m_den.copy()
    md[..., 1:] *= f[..., None]
    ed = e_den * f.reshape(e_den.shape[:2] + (1,) * (e_den.ndim - 2))
    return md, ed


def ensemble_decks(count: int = 256, seed: int = 2024, nmin: int = 128, nmax: int = 1024) -> List[Deck]:
    """Seeded ensemble of uneven impacts: grids drawn uniformly between nmin and nmax cells per
    axis, impactor speed U[5, 20] km/s, CPPR U{10..40}, cohesion log-uniform 1-100 MPa, friction
    U[0.6, 1.4]; basalt Tillotson target and projectile, 30-layer PML (at most a sixth of the mesh)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx = int(rng.integers(nmin, nmax + 1))
        ny = int(rng.integers(nmin, nmax + 1))
        v = float(rng.uniform(5000.0, 20000.0))
        cppr = int(rng.integers(10, 41))
        coh = float(10.0 ** rng.uniform(6.0, 8.0))
        fri = float(rng.uniform(0.6, 1.4))
        basalt = Material("basalt_", yint0=coh, yintfri=fri, ydam0=coh * 0.01, ydamfri=fri * 0.5)
        damp = max(4, min(30, min(nx, ny) // 6))
        out.append(Deck(npx=nx, npy=ny, dx=50.0, dy=50.0, oy=0.5, materials=[basalt], target_materials=["basalt_"],
                        target_depths=[1.0e7], projectile="basalt_", radius_cells=float(min(cppr, min(nx, ny) // 5)),
                        velocity=-v, gravity=-1.62, damping="pml", damp_x=damp, damp_y=damp, maxstep=1999,
                        dt0=1.0e-4, maxdt=0.05))
    return out


def config5_deck(n: int = 512, cohesion: float = 1.0e7, friction: float = 1.2, velocity: float = 8000.0,
                 cppr: float = 20.0, maxstep: int = 199) -> Deck:
    """n x n cells at 50 m, basalt Tillotson target and projectile (CPPR 20, 8 km/s), the
    Drucker-Prager parameters as RockStrengthT's intact and damaged cohesion (yint0 = ydam0),
    friction (yintfri = ydamfri) and limit 2.5 GPa, Ivanov damage, gravity. The deck of the
    adjoint window: no damping layers (the shock stays far from the boundaries over 200 cycles),
    numbers written exactly so that finite differences of a parameter reach the solver. The
    projectile starts at 1 MPa: at the default 1e-5 Pa its cells sit exactly at rho0 with a
    pressure below 0.01 Pa, on a node of the Tillotson cold-energy table and on the sound-speed
    switch of the EOS, kinks where the derivative is one-sided."""
    basalt = Material("basalt_", yint0=cohesion, yintfri=friction, yintlim=2.5e9, ydam0=cohesion,
                      ydamfri=friction, ydamlim=2.5e9)
    return Deck(npx=n, npy=n, dx=50.0, dy=50.0, oy=0.5, materials=[basalt], target_materials=["basalt_"],
                target_depths=[1.0e7], projectile="basalt_", radius_cells=cppr, velocity=-velocity, gravity=-1.62,
                damping="none", damp_x=0, damp_y=0, maxstep=maxstep, dt0=1.0e-4, maxdt=0.05, exact=True,
                projectile_pressure=1.0e6)


def target_profile(h0: np.ndarray, dx: float, seed: int = 5) -> np.ndarray:
    """Seeded target surface-height profile for the adjoint misfit: the initial material column
    heights h0 (one per interior column) with a Gaussian bowl cut out (depth U[200, 400] m, width
    U[20, 40] cells, centred on the axis) and +-1 m seeded roughness."""
    rng = np.random.default_rng(seed)
    depth = rng.uniform(200.0, 400.0)
    width = rng.uniform(20.0, 40.0) * dx
    r = (np.arange(len(h0)) + 0.5) * dx
    return h0 - depth * np.exp(-(r / width) ** 2) + rng.uniform(-1.0, 1.0, len(h0))
