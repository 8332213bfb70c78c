"""Host-side derivation of every engine constant + ctypes mirrors of the ABI.

The reference derives its per-step constants in Python inside the engine
constructors; they are float64 expressions evaluated by CPython.  This module
evaluates the same expressions in the same order, so the values handed to the
GPU are bit-identical to the reference's:

* DynamicsEngine.__init__   (ed_mrdt/dynamics.py:1724-2148)
* RateMatrix / _build_pss_matrices / PhotonSimulator.__init__
  (ed_mrdt/photophysics.py:59-151, 218-331, 690-1019)
* PSF / ConfocalScanner / TCSPCAccumulator / DetectorModel
  (ed_mrdt/microscope.py:73-285, 660-714, 830-837)

It also builds the exact Hill-factor tables: the reference's density value
in a grid cell holding k particles is the k-fold sequential float64 sum of
1/cell_area (dynamics.py:1697-1703), so the Hill factor is a function of the
integer count k and is tabulated here with the reference's own expression.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .config import ConfigError, SimulationConfig

MAX_SPECIES = 16
MAX_BIND = 4
MAX_CAT = 8
MAX_EXCH = 8
MAX_CONV = 8
MAX_GRIDS = 8
MAX_RULES = 24
MAX_REGIONS = 8
MAX_FLUO = 4
MAX_FRET = 4
MAX_FCLASS = 8

DFIELD_NONE, DFIELD_REGIONS, DFIELD_SINE_X = 0, 1, 2

# counters (enum EdmCounter)
(C_BINDINGS, C_DISSOC, C_CATALYTIC, C_RECRUITED, C_DETACHED, C_CONVERTED,
 C_PHOTONS, C_DONOR_PH, C_ACCEPTOR_PH, C_FRET_PH, C_DETECTED, C_DARK,
 C_AFTERPULSE, C_RECEIVED, NCOUNTERS) = range(15)


# ----------------------------------------------------------------------------
# ctypes mirrors of include/edm_b200.h (checked against edm_abi_sizeof)
# ----------------------------------------------------------------------------
class EdmGrid(C.Structure):
    _fields_ = [("sensor", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("pad", C.c_int32),
                ("sx", C.c_double), ("sy", C.c_double), ("offset", C.c_int64),
                ("inv_sx", C.c_double), ("inv_sy", C.c_double)]


class EdmRule(C.Structure):
    _fields_ = [("grid", C.c_int32), ("inhibition", C.c_int32), ("table_len", C.c_int32),
                ("pad", C.c_int32), ("table_offset", C.c_int64), ("K_half", C.c_double),
                ("n_hill", C.c_double), ("basal", C.c_double), ("inv_area", C.c_double)]


class EdmBind(C.Structure):
    _fields_ = [("ra", C.c_int32), ("rb", C.c_int32), ("product", C.c_int32), ("pad", C.c_int32),
                ("contact_sq", C.c_double), ("prob_bind", C.c_double), ("prob_dissoc", C.c_double)]


class EdmCat(C.Structure):
    _fields_ = [("enzyme", C.c_int32), ("substrate", C.c_int32), ("product", C.c_int32),
                ("rule", C.c_int32), ("contact_sq", C.c_double), ("prob", C.c_double)]


class EdmExch(C.Structure):
    _fields_ = [("species", C.c_int32), ("max_recruits", C.c_int32), ("rule_on", C.c_int32),
                ("rule_on2", C.c_int32), ("rule_off", C.c_int32), ("local_recruit", C.c_int32),
                ("prob_on", C.c_double), ("prob_off", C.c_double)]


class EdmConv(C.Structure):
    _fields_ = [("from_", C.c_int32), ("to", C.c_int32), ("rule", C.c_int32), ("pad", C.c_int32),
                ("prob", C.c_double)]


class EdmDynParams(C.Structure):
    _fields_ = [
        ("Lx", C.c_double), ("Ly", C.c_double), ("dt", C.c_double),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("cell_sx", C.c_double), ("cell_sy", C.c_double), ("cutoff_sq", C.c_double),
        ("particle_offset", C.c_int64), ("n_particles", C.c_int64),
        ("cell_offset", C.c_int64), ("grid_cells", C.c_int64),
        ("max_disp", C.c_double), ("max_disp_sq", C.c_double), ("force_range_sq", C.c_double),
        ("force_reach", C.c_double),
        ("use_wca", C.c_int32), ("use_harmonic", C.c_int32), ("n_species", C.c_int32),
        ("dfield", C.c_int32),
        ("D_base", C.c_double * MAX_SPECIES),
        ("sigma", C.c_double * (MAX_SPECIES * MAX_SPECIES)),
        ("eps", C.c_double * (MAX_SPECIES * MAX_SPECIES)),
        ("kharm", C.c_double * (MAX_SPECIES * MAX_SPECIES)),
        ("n_regions", C.c_int32), ("pad0", C.c_int32),
        ("reg_cx", C.c_double * MAX_REGIONS), ("reg_cy", C.c_double * MAX_REGIONS),
        ("reg_r", C.c_double * MAX_REGIONS), ("reg_f", C.c_double * MAX_REGIONS),
        ("smooth_w", C.c_double), ("sine_amp", C.c_double), ("sine_wavelength", C.c_double),
        ("n_bind", C.c_int32), ("n_cat", C.c_int32), ("n_exch", C.c_int32), ("n_conv", C.c_int32),
        ("n_grids", C.c_int32), ("n_rules", C.c_int32),
        ("bind", EdmBind * MAX_BIND), ("cat", EdmCat * MAX_CAT), ("exch", EdmExch * MAX_EXCH),
        ("conv", EdmConv * MAX_CONV), ("grid", EdmGrid * MAX_GRIDS), ("rule", EdmRule * MAX_RULES),
        ("adapt_grid", C.c_int32), ("adapt_cat_mask", C.c_int32),
        ("adapt_inv_tau", C.c_double), ("adapt_K", C.c_double), ("adapt_n", C.c_double),
        ("adapt_inv_area", C.c_double), ("recruit_sigma", C.c_double),
        ("seed", C.c_uint64),
    ]


class EdmFret(C.Structure):
    _fields_ = [("mode", C.c_int32), ("donor_fid", C.c_int32), ("acceptor_fid", C.c_int32),
                ("intramolecular", C.c_int32), ("cls_bound", C.c_int32), ("cls_high", C.c_int32),
                ("cls_low", C.c_int32), ("target_species", C.c_int32), ("prox_radius_sq", C.c_double)]


_T3 = ((C.c_double * MAX_FCLASS) * 2) * MAX_FLUO


# census row fields (EdmCensusField of include/edm_b200.h)
CEN_COUNTERS, CEN_BOND_ALIVE, CEN_BOND_ALL, CEN_BLEACHED, CEN_SPECIES = 0, 7, 8, 9, 10
CEN_DONORS, CEN_DONOR_CLS, CEN_FREE_DYE, CENSUS_FIELDS = 26, 27, 35, 40


class EdmPhotParams(C.Structure):
    _fields_ = [
        ("n_fluoro", C.c_int32), ("n_fret", C.c_int32),
        ("ground", C.c_int32 * MAX_FLUO), ("excited", C.c_int32 * MAX_FLUO),
        ("t1", C.c_int32 * MAX_FLUO), ("bl", C.c_int32 * MAX_FLUO),
        ("mean_d", _T3), ("mean_f", _T3), ("exp_neg_d", _T3), ("exp_neg_f", _T3),
        ("T00", _T3), ("T0001", _T3),
        ("tau", (C.c_double * MAX_FCLASS) * MAX_FLUO),
        ("fret_E", (C.c_double * MAX_FCLASS) * MAX_FLUO),
        ("gt_donor", C.c_int32 * MAX_FLUO),
        ("tau_all", C.c_double * MAX_FLUO),
        ("has_fret_cls", C.c_int32 * MAX_FCLASS),
        ("fret", EdmFret * MAX_FRET),
        ("donor_channel", C.c_int32), ("acceptor_channel", C.c_int32),
        ("max_photons", C.c_int64), ("est_photons", C.c_int64),
        ("photon_offset", C.c_int64), ("emitter_offset", C.c_int64), ("n_emitters", C.c_int64),
    ]


class EdmScopeParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("n_bins", C.c_int32), ("n_channels", C.c_int32),
        ("psf_range_px", C.c_int32), ("n_sigma", C.c_int32),
        ("pixel_size", C.c_double), ("offset_x", C.c_double), ("offset_y", C.c_double),
        ("bin_width", C.c_double), ("sigma_irf", C.c_double), ("qe", C.c_double),
        ("sigma_ch", C.c_double * MAX_FLUO), ("inv_2sig2_ch", C.c_double * MAX_FLUO),
        ("dark_lambda", C.c_double), ("dark_exp_neg", C.c_double), ("ap_prob", C.c_double),
        ("flim_offset", C.c_int64),
    ]


class EdmFlimParams(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("n_replicas", C.c_int32), ("n_emitters", C.c_int32),
                ("n_bins", C.c_int32), ("half_taps", C.c_int32), ("seed", C.c_uint64),
                ("bin_width_ns", C.c_double), ("sigma_irf_ns", C.c_double), ("sigma_psf_px", C.c_double),
                ("tau_free_ns", C.c_double), ("tau_bound_ns", C.c_double),
                ("yield_free", C.c_double), ("yield_bound", C.c_double)]


class EdmHostState(C.Structure):
    _fields_ = [("n", C.c_int64), ("positions", C.c_void_p), ("species_id", C.c_void_p),
                ("is_alive", C.c_void_p), ("bond_partner", C.c_void_p), ("has_dye", C.c_void_p),
                ("dye_type_id", C.c_void_p), ("ctmc_state", C.c_void_p), ("is_bleached", C.c_void_p)]


# ----------------------------------------------------------------------------
# Dynamics constants (dynamics.py:1724-2148)
# ----------------------------------------------------------------------------
def _hill_value(rho: float, K_half: float, n_hill: float, inhibition: bool, basal: float) -> float:
    """The Hill factor exactly as inlined in the reference kernels
    (e.g. dynamics.py:965-976)."""
    if K_half > 0:
        ratio = rho / K_half
        ratio_n = ratio ** n_hill
        if inhibition:
            return 1.0 / (1.0 + ratio_n)
        h = ratio_n / (1.0 + ratio_n)
        return basal + (1.0 - basal) * h
    return 1.0


def hill_table(inv_area: float, K_half: float, n_hill: float, inhibition: bool, basal: float,
               length: int) -> np.ndarray:
    """Hill factor for integer counts 0..length-1, with the density of k
    particles formed as the reference does: k sequential float64 additions of
    inv_area starting from 0.0 (dynamics.py:1697-1703)."""
    out = np.empty(length, dtype=np.float64)
    rho = 0.0
    for k in range(length):
        out[k] = _hill_value(rho, K_half, n_hill, inhibition, basal)
        rho = rho + inv_area
    return out


@dataclass
class DynDerived:
    """Constants of one replica, by name, for tests and host logic."""
    cutoff_um: float = 0.0
    nx: int = 0
    ny: int = 0
    cell_sx: float = 0.0
    cell_sy: float = 0.0
    max_displacement: float = 0.0
    use_wca: bool = False
    use_harmonic: bool = False
    sigma_matrix: Optional[np.ndarray] = None
    epsilon_matrix: Optional[np.ndarray] = None
    harmonic_matrix: Optional[np.ndarray] = None
    reactions: List[dict] = field(default_factory=list)
    catalytic: List[dict] = field(default_factory=list)
    exchanges: List[dict] = field(default_factory=list)
    conversions: List[dict] = field(default_factory=list)
    grids: List[Tuple] = field(default_factory=list)
    rules: List[Tuple] = field(default_factory=list)
    # adaptation field (dynamics.py:2078-2096): grid index (-1 off), modulated catalytic reactions
    adapt_grid: int = -1
    adapt_cat_mask: int = 0
    adapt_inv_tau: float = 0.0
    adapt_K: float = 0.0
    adapt_n: float = 0.0
    adapt_inv_area: float = 0.0
    recruit_sigma: float = 0.5


def derive_dynamics(config: SimulationConfig) -> DynDerived:
    """Every DynamicsEngine.__init__ constant (dynamics.py:1724-2148)."""
    d = DynDerived()
    Lx, Ly = config.membrane.size
    dt = config.bd_timestep
    names = {s.name: i for i, s in enumerate(config.species)}
    spec = config.species

    # cutoff (dynamics.py:1738-1782)
    max_nm = config.max_potential_cutoff
    for rx in config.reactions:
        if rx.contact_radius > max_nm:
            max_nm = rx.contact_radius
    for cat in config.catalytic_reactions:
        if cat.contact_radius > max_nm:
            max_nm = cat.contact_radius
    max_um = max_nm / 1000.0
    for rx in config.reactions:
        if rx.is_bimolecular and rx.kon > 0:
            a, b = names[rx.reactants[0]], names[rx.reactants[1]]
            s_bd = math.sqrt(4.0 * (spec[a].diffusion_coefficient + spec[b].diffusion_coefficient) * dt)
            eff = max(rx.contact_radius / 1000.0, s_bd)
            if eff > max_um:
                max_um = eff
    for cat in config.catalytic_reactions:
        a, b = names[cat.enzyme], names[cat.substrate]
        s_bd = math.sqrt(4.0 * (spec[a].diffusion_coefficient + spec[b].diffusion_coefficient) * dt)
        eff = max(cat.contact_radius / 1000.0, s_bd)
        if eff > max_um:
            max_um = eff
    cutoff = max(max_um, max_nm / 1000.0) * 1.1
    if cutoff < 0.001:
        cutoff = 0.05
    if cutoff <= 0:
        raise ValueError(f"cutoff must be positive, got {cutoff}")
    d.cutoff_um = cutoff
    # cell grid (dynamics.py:109-114)
    d.nx = max(3, int(math.floor(Lx / cutoff)))
    d.ny = max(3, int(math.floor(Ly / cutoff)))
    d.cell_sx = Lx / d.nx
    d.cell_sy = Ly / d.ny

    # potentials (dynamics.py:1790-1824)
    n_sp = config.n_species
    sig = np.zeros((n_sp, n_sp))
    eps = np.zeros((n_sp, n_sp))
    kh = np.zeros((n_sp, n_sp))
    for pot in config.potentials:
        a, b = names[pot.species_a], names[pot.species_b]
        if pot.potential_type in ("wca", "lennard_jones"):
            d.use_wca = True
            s_um = pot.parameters.get("sigma", 5.0) / 1000.0
            e = pot.parameters.get("epsilon", 2.5)
            sig[a, b] = sig[b, a] = s_um
            eps[a, b] = eps[b, a] = e
        elif pot.potential_type == "harmonic_repulsion":
            d.use_harmonic = True
            s_um = pot.parameters.get("sigma", 5.0) / 1000.0
            k = pot.parameters.get("spring_constant", pot.parameters.get("epsilon", 50.0))
            sig[a, b] = sig[b, a] = s_um
            kh[a, b] = kh[b, a] = k
    d.sigma_matrix, d.epsilon_matrix, d.harmonic_matrix = sig, eps, kh

    # displacement cap (dynamics.py:1837-1864)
    sigma_min = np.inf
    for i in range(n_sp):
        for j in range(n_sp):
            if sig[i, j] > 0:
                sigma_min = min(sigma_min, sig[i, j])
    D_max = max(s.diffusion_coefficient for s in spec)
    contact_max = 0.0
    for cat in config.catalytic_reactions:
        contact_max = max(contact_max, cat.contact_radius / 1000.0)
    if d.use_wca:
        d.max_displacement = max(config.displacement_cap_fraction * sigma_min, contact_max)
    elif d.use_harmonic:
        rms = np.sqrt(2.0 * D_max * config.bd_timestep)
        d.max_displacement = max(5.0 * rms, contact_max, sigma_min if sigma_min < np.inf else 0.1)
    elif sigma_min < np.inf:
        d.max_displacement = config.displacement_cap_fraction * sigma_min
    else:
        d.max_displacement = 0.1
    d.max_displacement = float(d.max_displacement)

    # binding (dynamics.py:1866-1952)
    for rx in config.reactions:
        if not rx.is_bimolecular:
            continue
        a, b = names[rx.reactants[0]], names[rx.reactants[1]]
        prod = names[rx.products[0]]
        contact = rx.contact_radius / 1000.0
        D_rel = spec[a].diffusion_coefficient + spec[b].diffusion_coefficient
        s_bd = math.sqrt(4.0 * D_rel * dt)
        eff = max(contact, s_bd)
        A_eff = math.pi * (eff ** 2)
        if A_eff > 0 and rx.kon > 0:
            kon = rx.kon
            N_b = config.initial_populations.get(rx.reactants[1], 0)
            area = config.membrane.size[0] * config.membrane.size[1]
            c_b = N_b / area if area > 0 else 0
            L_half = min(config.membrane.size) / 2.0
            if c_b > 0 and D_rel > 0 and contact > 0:
                R_ck = min(1.0 / math.sqrt(math.pi * c_b), L_half)
                ln_ratio = math.log(R_ck / contact)
                if ln_ratio > 0:
                    inv_k = 1.0 / kon - ln_ratio / (2.0 * math.pi * D_rel)
                    k_int = 1.0 / inv_k if inv_k > 0 else 1e12
                    p_bind = min(1.0, k_int * dt / A_eff)
                else:
                    p_bind = min(1.0, kon * dt / A_eff)
            else:
                p_bind = min(1.0, kon * dt / A_eff)
        else:
            p_bind = 0.0
        d.reactions.append(dict(ra=a, rb=b, product=prod, contact_um=eff, prob_bind=p_bind,
                                prob_dissoc=min(1.0, rx.koff * dt)))

    fbmap = {fb.name: fb for fb in config.feedback_rules}

    def grid_of(fb) -> Tuple:
        nxg = max(3, int(Lx / fb.grid_resolution))
        nyg = max(3, int(Ly / fb.grid_resolution))
        return (names[fb.sensor_species], nxg, nyg, Lx / nxg, Ly / nyg)

    def rule_of(name: Optional[str]) -> int:
        if not name or name not in fbmap:
            return -1
        fb = fbmap[name]
        g = grid_of(fb)
        if g not in d.grids:
            d.grids.append(g)
        key = (d.grids.index(g), fb.function_type == "hill_inhibition", fb.K_half, fb.n_hill,
               fb.basal_fraction)
        if key not in d.rules:
            d.rules.append(key)
        return d.rules.index(key)

    # catalytic (dynamics.py:1979-2008)
    for cat in config.catalytic_reactions:
        e, s, p = names[cat.enzyme], names[cat.substrate], names[cat.product]
        D_rel = spec[e].diffusion_coefficient + spec[s].diffusion_coefficient
        contact = cat.contact_radius / 1000.0
        s_bd = math.sqrt(4.0 * D_rel * dt)
        eff = max(contact, s_bd)
        A_eff = math.pi * eff ** 2
        prob = min(1.0, cat.k_cat * dt / max(A_eff, 1e-30))
        d.catalytic.append(dict(enzyme=e, substrate=s, product=p, contact_um=eff, prob=prob,
                                rule=rule_of(cat.feedback_rule)))
    # exchanges (dynamics.py:2010-2043)
    for ex in config.compartment_exchanges:
        r_on = rule_of(ex.feedback_rule)
        r_on2 = rule_of(ex.secondary_feedback_rule)
        d.exchanges.append(dict(species=names[ex.species], prob_on=min(1.0, ex.k_on * dt),
                                prob_off=min(1.0, ex.k_off * dt),
                                max_recruits=int(ex.max_recruits_per_step),
                                rule_on=r_on, rule_on2=r_on2 if r_on >= 0 else -1,
                                rule_off=rule_of(ex.detachment_feedback_rule)))
    # conversions (dynamics.py:2046-2065)
    for cv in config.unimolecular_conversions:
        d.conversions.append(dict(from_id=names[cv.from_species], to_id=names[cv.to_species],
                                  prob=min(1.0, cv.rate * dt), rule=rule_of(cv.feedback_rule)))

    # local (density-biased) recruitment (dynamics.py:2029-2045, 2116-2120, 2354): exchanges with a
    # single feedback rule whose name holds 'pip3_activation'
    use_local = bool(getattr(config, "use_local_pi3k_recruitment", False))
    d.recruit_sigma = float(getattr(config, "recruit_sigma", 0.5))
    for ex, r in zip(config.compartment_exchanges, d.exchanges):
        r["local"] = int(use_local and bool(ex.feedback_rule) and "pip3_activation" in ex.feedback_rule
                         and r["rule_on"] >= 0 and r["rule_on2"] < 0)

    # adaptation field (dynamics.py:2078-2096, 1998-2007): a 1 µm grid of PIP3 density relaxed with
    # tau_w; catalytic reactions whose enzyme name holds 'PI3K' (and that have feedback) are
    # modulated by 1/(1 + (w/K)^n), w read at the feedback grid's (gx, gy)
    if getattr(config, "use_adaptation", False):
        anx, any_ = max(3, int(Lx / 1.0)), max(3, int(Ly / 1.0))
        asx, asy = Lx / anx, Ly / any_
        pip3 = names.get("PIP3", -1)
        if pip3 >= 0:
            g = (pip3, anx, any_, asx, asy)
            if g not in d.grids:
                d.grids.append(g)
            d.adapt_grid = d.grids.index(g)
        d.adapt_inv_tau = dt / float(getattr(config, "adaptation_tau_w", 60.0))
        d.adapt_K = float(getattr(config, "adaptation_K_w", 10.0))
        d.adapt_n = float(getattr(config, "adaptation_n_w", 2.0))
        area = asx * asy
        d.adapt_inv_area = 1.0 / area if area > 0.0 else 0.0
        for k, (cat, r) in enumerate(zip(config.catalytic_reactions, d.catalytic)):
            if "PI3K" in cat.enzyme and r["rule"] >= 0:
                _, fnx, fny, _, _ = d.grids[d.rules[r["rule"]][0]]
                # the reference reads adaptation_field[gx, gy] with the feedback grid's (gx, gy): past
                # its (anx, any_) array when the feedback grid is larger (undefined memory there)
                if (fnx - 1) * any_ + (fny - 1) >= anx * any_:
                    raise NotImplementedError(
                        f"adaptation of catalytic reaction '{cat.name}': its feedback grid ({fnx}x{fny}) is larger "
                        f"than the 1 µm adaptation grid ({anx}x{any_}); the reference then reads past the "
                        "adaptation array (dynamics.py:1078). Use a 1 µm feedback grid_resolution.")
                d.adapt_cat_mask |= 1 << k
    return d


def force_range_sq(d: DynDerived) -> float:
    """Largest squared separation at which any pair force is non-zero: the
    WCA range 2^(1/3) sigma^2 (dynamics.py:711) or the harmonic sigma^2
    (dynamics.py:796), evaluated with the kernels' own expressions."""
    best = 0.0
    n = d.sigma_matrix.shape[0]
    for i in range(n):
        for j in range(n):
            sig = float(d.sigma_matrix[i, j])
            if sig <= 0.0:
                continue
            if d.use_wca and d.epsilon_matrix[i, j] > 0.0:
                best = max(best, sig * sig * 1.2599210498948732)
            if d.use_harmonic and d.harmonic_matrix[i, j] > 0.0:
                best = max(best, sig * sig)
    return best


def n_buckets(d: DynDerived) -> int:
    """Sort buckets of one replica: its cells plus one for non-alive particles."""
    return d.nx * d.ny + 1


def check_supported(config: SimulationConfig) -> None:
    """Features of the reference outside this engine raise here, loudly."""
    if config.n_species > MAX_SPECIES:
        raise ConfigError(f"at most {MAX_SPECIES} species")
    for cat in config.catalytic_reactions:
        if cat.product == cat.enzyme or cat.enzyme == cat.substrate:
            raise NotImplementedError(
                f"catalytic reaction '{cat.name}': enzyme == product/substrate makes a pass "
                "order-dependent; not supported by the parallel pass")
    enzymes = {c.enzyme for c in config.catalytic_reactions}
    converted = {c.substrate for c in config.catalytic_reactions} | {c.product for c in config.catalytic_reactions}
    if enzymes & converted:
        raise NotImplementedError(
            f"species {sorted(enzymes & converted)} are both enzymes and catalytic substrates/products; "
            "the per-step contact list requires enzymes to keep their species during the catalytic passes")
    for rx in config.reactions:
        if rx.is_bimolecular and rx.products and rx.products[0] in rx.reactants:
            raise NotImplementedError(
                f"binding reaction '{rx.name}': a product equal to a reactant re-enters the same pass; "
                "not supported by the candidate-list pass")
    df = config.diffusion_field
    if df.type not in ("uniform", "regions", "sine_x"):
        raise NotImplementedError(f"diffusion_field.type '{df.type}'")


def build_dyn_params(config: SimulationConfig, n_particles: int, seed: Optional[int] = None,
                     hill_len: Optional[int] = None, particle_offset: int = 0, cell_offset: int = 0,
                     grid_offset: int = 0, hill_offset: int = 0
                     ) -> Tuple[EdmDynParams, np.ndarray, DynDerived]:
    """Fill one replica's EdmDynParams and its Hill tables.

    hill_len: entries per exact Hill table (default n_particles + 1, i.e.
    complete: a grid cell cannot hold more particles than exist).
    Offsets place this replica's slices in the engine's global arrays.
    """
    check_supported(config)
    d = derive_dynamics(config)
    if len(d.reactions) > MAX_BIND or len(d.catalytic) > MAX_CAT or len(d.exchanges) > MAX_EXCH \
            or len(d.conversions) > MAX_CONV or len(d.grids) > MAX_GRIDS or len(d.rules) > MAX_RULES:
        raise ConfigError("too many reactions / feedback rules for the fixed parameter block")
    P = EdmDynParams()
    Lx, Ly = config.membrane.size
    P.Lx, P.Ly, P.dt = float(Lx), float(Ly), float(config.bd_timestep)
    P.periodic_x, P.periodic_y = int(bool(config.membrane.periodic[0])), int(bool(config.membrane.periodic[1]))
    P.nx, P.ny = d.nx, d.ny
    P.cell_sx, P.cell_sy = d.cell_sx, d.cell_sy
    P.cutoff_sq = d.cutoff_um * d.cutoff_um
    P.particle_offset, P.n_particles, P.cell_offset = particle_offset, n_particles, cell_offset
    P.max_disp = d.max_displacement
    P.max_disp_sq = d.max_displacement * d.max_displacement
    P.force_range_sq = force_range_sq(d)
    P.force_reach = math.sqrt(min(P.force_range_sq, P.cutoff_sq)) * 1.0001 + 1e-9
    P.use_wca, P.use_harmonic, P.n_species = int(d.use_wca), int(d.use_harmonic), config.n_species
    for i, s in enumerate(config.species):
        P.D_base[i] = s.diffusion_coefficient
    n_sp = config.n_species
    for i in range(n_sp):
        for j in range(n_sp):
            P.sigma[i * MAX_SPECIES + j] = d.sigma_matrix[i, j]
            P.eps[i * MAX_SPECIES + j] = d.epsilon_matrix[i, j]
            P.kharm[i * MAX_SPECIES + j] = d.harmonic_matrix[i, j]
    df = config.diffusion_field
    circles = [r for r in df.regions if r.get("shape") == "circle"]
    if df.type == "sine_x":
        P.dfield = DFIELD_SINE_X
        P.sine_amp, P.sine_wavelength = float(df.amplitude), float(df.wavelength)
    elif circles:
        if len(circles) > MAX_REGIONS:
            raise ConfigError(f"at most {MAX_REGIONS} D-field regions")
        P.dfield = DFIELD_REGIONS
        P.n_regions = len(circles)
        for k, r in enumerate(circles):
            P.reg_cx[k], P.reg_cy[k] = float(r["center"][0]), float(r["center"][1])
            P.reg_r[k], P.reg_f[k] = float(r["radius"]), float(r.get("D_factor", 1.0))
    else:
        P.dfield = DFIELD_NONE
    P.smooth_w = float(config.region_smoothing_width)

    P.n_bind = len(d.reactions)
    for k, r in enumerate(d.reactions):
        b = P.bind[k]
        b.ra, b.rb, b.product = r["ra"], r["rb"], r["product"]
        b.contact_sq = r["contact_um"] * r["contact_um"]
        b.prob_bind, b.prob_dissoc = r["prob_bind"], r["prob_dissoc"]
    P.n_cat = len(d.catalytic)
    for k, r in enumerate(d.catalytic):
        c = P.cat[k]
        c.enzyme, c.substrate, c.product, c.rule = r["enzyme"], r["substrate"], r["product"], r["rule"]
        c.contact_sq = r["contact_um"] * r["contact_um"]
        c.prob = r["prob"]
    P.n_exch = len(d.exchanges)
    for k, r in enumerate(d.exchanges):
        e = P.exch[k]
        e.species, e.max_recruits = r["species"], r["max_recruits"]
        e.rule_on, e.rule_on2, e.rule_off = r["rule_on"], r["rule_on2"], r["rule_off"]
        e.local_recruit = r["local"]
        e.prob_on, e.prob_off = r["prob_on"], r["prob_off"]
    P.n_conv = len(d.conversions)
    for k, r in enumerate(d.conversions):
        v = P.conv[k]
        v.from_, v.to, v.rule, v.prob = r["from_id"], r["to_id"], r["rule"], r["prob"]

    P.n_grids = len(d.grids)
    goff = grid_offset
    for k, (sensor, nxg, nyg, sx, sy) in enumerate(d.grids):
        g = P.grid[k]
        g.sensor, g.nx, g.ny, g.sx, g.sy, g.offset = sensor, nxg, nyg, sx, sy, goff
        g.inv_sx, g.inv_sy = 1.0 / sx, 1.0 / sy
        goff += nxg * nyg
    P.grid_cells = goff - grid_offset
    tlen = int(hill_len) if hill_len is not None else n_particles + 1
    tables = []
    P.n_rules = len(d.rules)
    hoff = hill_offset
    for k, (gi, inhib, K, n, basal) in enumerate(d.rules):
        _, _, _, sx, sy = d.grids[gi]
        area = sx * sy
        inv_area = 1.0 / area if area > 0.0 else 0.0
        R = P.rule[k]
        R.grid, R.inhibition, R.table_len, R.table_offset = gi, int(inhib), tlen, hoff
        R.K_half, R.n_hill, R.basal, R.inv_area = K, n, basal, inv_area
        tables.append(hill_table(inv_area, K, n, inhib, basal, tlen))
        hoff += tlen
    P.adapt_grid, P.adapt_cat_mask = d.adapt_grid, d.adapt_cat_mask
    P.adapt_inv_tau, P.adapt_K, P.adapt_n = d.adapt_inv_tau, d.adapt_K, d.adapt_n
    P.adapt_inv_area, P.recruit_sigma = d.adapt_inv_area, d.recruit_sigma
    P.seed = int(config.random_seed if seed is None else seed) & 0xFFFFFFFFFFFFFFFF
    hill = np.concatenate(tables) if tables else np.zeros(0, dtype=np.float64)
    return P, hill, d


# ----------------------------------------------------------------------------
# Photophysics constants (photophysics.py:59-151, 218-331, 690-1019)
# ----------------------------------------------------------------------------
class _Rates:
    """Rate-matrix quantities of one fluorophore (photophysics.py:59-151)."""

    def __init__(self, fluo):
        self.fluo = fluo
        n = fluo.n_states
        self.n_states = n
        smap = {s.name: i for i, s in enumerate(fluo.states)}
        Q = np.zeros((n, n), dtype=np.float64)
        for src, dsts in fluo.thermal_rates.items():
            for dst, rate in dsts.items():
                Q[smap[src], smap[dst]] = rate
        for i in range(n):
            Q[i, i] = 0.0
            Q[i, i] = -np.sum(Q[i, :])
        self.Q = Q
        self.exit_rates = np.zeros(n)
        self.branch = np.zeros((n, n))
        for i in range(n):
            tot = -Q[i, i]
            self.exit_rates[i] = tot
            if tot > 0:
                for j in range(n):
                    if j != i:
                        self.branch[i, j] = Q[i, j] / tot
        st = fluo.states
        self.ground = next((i for i, s in enumerate(st) if s.is_absorbing and not s.is_fluorescent), 0)
        self.excited = next((i for i, s in enumerate(st) if s.is_fluorescent), -1)
        self.t1 = next((i for i, s in enumerate(st)
                        if not s.is_absorbing and not s.is_fluorescent and not s.is_terminal), -1)
        self.bl = next((i for i, s in enumerate(st) if s.is_terminal), -1)

    def lifetime(self, state: int) -> float:
        k = self.exit_rates[state]
        return float("inf") if k <= 0 else 1.0 / k


def _pss(rm: _Rates, p_exc: float, T_laser: float, n_pulses: int, k_fret: float = 0.0,
         QY_d: float = 1.0, QY_a: float = 1.0) -> Dict:
    """Per-BD-step Poisson-steady-state matrices (photophysics.py:218-331)."""
    s0, s1, t1, bl = rm.ground, rm.excited, rm.t1, rm.bl
    kS1 = rm.exit_rates[s1] + k_fret if (k_fret > 0 and s1 >= 0) else rm.exit_rates[s1]
    if kS1 > 0 and s1 >= 0:
        p_rad = rm.Q[s1, s0] / kS1
        p_fr = k_fret / kS1 if k_fret > 0 else 0.0
        p_isc = rm.Q[s1, t1] / kS1 if t1 >= 0 else 0.0
        p_bl = rm.Q[s1, bl] / kS1 if bl >= 0 else 0.0
    else:
        p_rad = p_fr = p_isc = p_bl = 0.0
    p_back = p_rad + p_fr
    if t1 >= 0:
        kT1 = rm.exit_rates[t1]
        p_exit = 1.0 - math.exp(-kT1 * T_laser) if kT1 > 0 else 0.0
        p_t1_s0 = rm.branch[t1, s0]
        p_t1_bl = rm.branch[t1, bl] if bl >= 0 else 0.0
    else:
        p_exit = p_t1_s0 = p_t1_bl = 0.0
    T = np.zeros((3, 3), dtype=np.float64)
    T[0, 0] = (1.0 - p_exc) + p_exc * p_back
    T[0, 1] = p_exc * p_isc
    T[0, 2] = p_exc * p_bl
    T[1, 0] = p_exit * p_t1_s0
    T[1, 1] = 1.0 - p_exit
    T[1, 2] = p_exit * p_t1_bl
    T[2, 2] = 1.0
    for r in range(3):
        rs = T[r].sum()
        if abs(rs - 1.0) > 1e-12:
            T[r] /= rs
    T_step = np.linalg.matrix_power(T, n_pulses)
    Ts = T[:2, :2].copy()
    I2 = np.eye(2, dtype=np.float64)
    Tn = np.linalg.matrix_power(Ts, n_pulses)
    try:
        S = (I2 - Tn) @ np.linalg.inv(I2 - Ts)
    except np.linalg.LinAlgError:
        S = np.zeros((2, 2))
        Tk = I2.copy()
        for _ in range(n_pulses):
            S += Tk
            Tk = Tk @ Ts
    p_d = p_exc * p_rad * QY_d
    mean_ph = np.zeros(2) if p_d <= 0.0 else np.array([S[0, 0] * p_d, S[1, 0] * p_d])
    p_f = p_exc * p_fr * QY_a
    mean_fret = np.zeros(2) if p_f <= 0.0 else np.array([S[0, 0] * p_f, S[1, 0] * p_f])
    tau = 1.0 / kS1 if kS1 > 0 else 4.1e-9
    return {"T_step": T_step, "mean_ph": mean_ph, "mean_fret": mean_fret, "tau_eff": tau}


def _excitation_prob(config: SimulationConfig, fluo) -> float:
    """Single-pulse excitation probability (photophysics.py:953-991)."""
    h = 6.626e-34
    c = 3.0e8
    las = config.laser
    E_ph = h * c / (las.wavelength * 1e-9)
    w0 = las.beam_waist * 1e-9
    A = math.pi * w0 ** 2
    n_pp = (las.power / las.repetition_rate) / E_ph
    flux = n_pp / A
    sig = fluo.absorption_cross_section * 1e-4
    if fluo.excitation_wavelength > 0:
        dl = abs(las.wavelength - fluo.excitation_wavelength)
        if dl > 1.0:
            fwhm = getattr(fluo, "absorption_fwhm", 45.0)
            sig *= math.exp(-0.5 * (dl / (fwhm / 2.355)) ** 2)
    return min(sig * flux, 0.9)


@dataclass
class PhotDerived:
    n_fluoro: int = 0
    active: bool = False
    rates: List[_Rates] = field(default_factory=list)
    n_pulses: int = 0
    laser_period: float = 0.0
    p_exc: Optional[np.ndarray] = None
    QY: Optional[np.ndarray] = None
    T_step: Optional[np.ndarray] = None
    T_step_fret: Optional[np.ndarray] = None
    mean_ph: Optional[np.ndarray] = None
    mean_ph_fret: Optional[np.ndarray] = None
    mean_fret: Optional[np.ndarray] = None
    mean_fret_fret: Optional[np.ndarray] = None
    tau_all: Optional[np.ndarray] = None
    tau_fret_all: Optional[np.ndarray] = None
    k_fret_bound: Optional[np.ndarray] = None
    fret_maps: List[dict] = field(default_factory=list)
    bond_pairs: List[dict] = field(default_factory=list)
    prox_pairs: List[dict] = field(default_factory=list)
    donor_channel: int = 0
    acceptor_channel: int = 1
    max_photons: int = 1000
    est_photons: int = 1000


def derive_photophysics(config: SimulationConfig, n_particles: int, n_labeled: int,
                        scan_duty_fraction: float) -> PhotDerived:
    """PhotonSimulator.__init__ constants (photophysics.py:693-887, 911-1114)."""
    d = PhotDerived()
    d.rates = [_Rates(f) for f in config.fluorophores]
    nf = len(d.rates)
    d.n_fluoro = nf
    if nf == 0:
        return d
    d.active = True
    duty = max(0.0, min(1.0, scan_duty_fraction))
    d.laser_period = config.laser.period
    d.n_pulses = max(1, int(round(config.bd_timestep / d.laser_period)))
    d.p_exc = np.array([_excitation_prob(config, f) for f in config.fluorophores])
    smap = {s.name: i for i, s in enumerate(config.species)}
    fmap = {f.name: i for i, f in enumerate(config.fluorophores)}
    for fp in config.fret_pairs:
        d.fret_maps.append(dict(R0=fp.R0, icd=fp.intra_complex_distance,
                                donor=fmap.get(fp.donor_type, -1),
                                acceptor=fmap.get(fp.acceptor_type, -1), cfg=fp))
    if d.fret_maps:
        d.donor_channel = d.fret_maps[0]["donor"]
        d.acceptor_channel = d.fret_maps[0]["acceptor"]
    else:
        d.donor_channel, d.acceptor_channel = 0, (1 if nf > 1 else 0)

    def pair_cfg(fm):
        for fp in config.fret_pairs:
            if fmap.get(fp.donor_type, -1) == fm["donor"] and fmap.get(fp.acceptor_type, -1) == fm["acceptor"]:
                return fp
        return None

    def bound_rate(t: int) -> float:
        for fm in d.fret_maps:
            if fm["donor"] == t:
                fp = pair_cfg(fm)
                rm = d.rates[t]
                tauD = rm.lifetime(rm.excited)
                if tauD <= 0 or math.isinf(tauD):
                    return 0.0
                if fp and getattr(fp, "fret_mode", "bond") == "proximity":
                    E = fp.proximity_E_high
                    return 1e15 if E >= 1.0 else E / ((1.0 - E) * tauD)
                ratio = fm["R0"] / fm["icd"]
                return ratio ** 6 / tauD
        return 0.0

    d.QY = np.ones(nf)
    for t, rm in enumerate(d.rates):
        if rm.excited >= 0:
            d.QY[t] = rm.fluo.states[rm.excited].quantum_yield
    d.T_step = np.zeros((nf, 3, 3)); d.T_step_fret = np.zeros((nf, 3, 3))
    d.mean_ph = np.zeros((nf, 2)); d.mean_ph_fret = np.zeros((nf, 2))
    d.mean_fret = np.zeros((nf, 2)); d.mean_fret_fret = np.zeros((nf, 2))
    d.tau_all = np.zeros(nf); d.tau_fret_all = np.zeros(nf); d.k_fret_bound = np.zeros(nf)
    for t, rm in enumerate(d.rates):
        p_exc = d.p_exc[t] * duty
        QY_d = float(d.QY[t])
        QY_a = 1.0
        for fm in d.fret_maps:
            if fm["donor"] == t:
                if 0 <= fm["acceptor"] < nf:
                    QY_a = float(d.QY[fm["acceptor"]])
                break
        base = _pss(rm, p_exc, d.laser_period, d.n_pulses, 0.0, QY_d, QY_a)
        d.T_step[t], d.mean_ph[t], d.mean_fret[t], d.tau_all[t] = \
            base["T_step"], base["mean_ph"], base["mean_fret"], base["tau_eff"]
        kb = bound_rate(t)
        d.k_fret_bound[t] = kb
        fr = _pss(rm, p_exc, d.laser_period, d.n_pulses, kb, QY_d, QY_a) if kb > 0 else base
        d.T_step_fret[t], d.mean_ph_fret[t], d.mean_fret_fret[t], d.tau_fret_all[t] = \
            fr["T_step"], fr["mean_ph"], fr["mean_fret"], fr["tau_eff"]

    # FRET pairs as evaluated by update_fret_rates (photophysics.py:1021-1114)
    for fm in d.fret_maps:
        fp = pair_cfg(fm)
        if fp and getattr(fp, "fret_mode", "bond") == "proximity":
            continue
        if fm["donor"] < 0 or fm["donor"] >= nf:
            continue
        rm = d.rates[fm["donor"]]
        tauD = rm.lifetime(rm.excited)
        if tauD <= 0 or math.isinf(tauD):
            continue
        ratio = fm["R0"] / fm["icd"]
        r6 = ratio * ratio * ratio * ratio * ratio * ratio
        d.bond_pairs.append(dict(R0=fm["R0"], tauD=tauD, icd=fm["icd"], donor=fm["donor"],
                                 acceptor=fm["acceptor"], k=r6 / tauD,
                                 intra=bool(getattr(fp, "intramolecular", False)) if fp else False))
    for fp in config.fret_pairs:
        if getattr(fp, "fret_mode", "bond") != "proximity":
            continue
        donor = fmap.get(fp.donor_type, -1)
        if donor < 0 or donor >= nf:
            continue
        rm = d.rates[donor]
        tauD = rm.lifetime(rm.excited)
        if tauD <= 0 or math.isinf(tauD):
            continue
        target = smap.get(fp.proximity_target_species, -1)
        if target < 0:
            continue
        Eh, El = fp.proximity_E_high, fp.proximity_E_low
        kh = Eh / ((1.0 - Eh) * tauD) if Eh < 1.0 else 1e15
        kl = El / ((1.0 - El) * tauD) if El < 1.0 else 1e15
        d.prox_pairs.append(dict(donor=donor, target=target, radius_um=fp.proximity_radius * 1e-3,
                                 k_high=kh, k_low=kl, tauD=tauD))

    max_mean = 0.0
    for t in range(nf):
        max_mean = max(max_mean, float(d.mean_ph[t, 0]))
    d.max_photons = max(1000, int(n_labeled * max_mean * 3))
    mm = 0.0
    for t in range(nf):
        mm = max(mm, max(float(d.mean_ph[t, 0]), float(d.mean_ph_fret[t, 0])))
    d.est_photons = max(1000, int(n_particles * mm * 2.5))
    return d


def build_phot_params(config: SimulationConfig, n_particles: int, n_labeled: int,
                      scan_duty_fraction: float, photon_offset: int = 0, emitter_offset: int = 0,
                      n_emitters: int = 0) -> Tuple[EdmPhotParams, PhotDerived]:
    """EdmPhotParams with the per-(dye, pss, FRET class) tables of the PSS
    kernel (photophysics.py:390-431) precomputed with the kernel's own
    float64 expressions, and exp(-mean) from the host libm as the kernel's
    math.exp would give."""
    d = derive_photophysics(config, n_particles, n_labeled, scan_duty_fraction)
    P = EdmPhotParams()
    P.n_fluoro = d.n_fluoro
    if not d.active:
        return P, d
    if d.n_fluoro > MAX_FLUO:
        raise ConfigError(f"at most {MAX_FLUO} fluorophores")
    # FRET classes: 0 = no FRET, then one per bond pair, two per proximity pair
    ks = [0.0]
    P.n_fret = 0
    for bp in d.bond_pairs:
        f = P.fret[P.n_fret]
        f.mode, f.donor_fid, f.acceptor_fid, f.intramolecular = 0, bp["donor"], bp["acceptor"], int(bp["intra"])
        f.cls_bound = len(ks); ks.append(bp["k"])
        f.cls_high = f.cls_low = 0
        f.target_species = -1
        P.n_fret += 1
    for pp in d.prox_pairs:
        f = P.fret[P.n_fret]
        f.mode, f.donor_fid, f.acceptor_fid, f.intramolecular = 1, pp["donor"], -1, 0
        f.cls_high = len(ks); ks.append(pp["k_high"])
        f.cls_low = len(ks); ks.append(pp["k_low"])
        f.cls_bound = 0
        f.target_species = pp["target"]
        f.prox_radius_sq = pp["radius_um"] * pp["radius_um"]
        P.n_fret += 1
    if len(ks) > MAX_FCLASS or P.n_fret > MAX_FRET:
        raise ConfigError("too many FRET pairs for the fixed parameter block")
    for t in range(d.n_fluoro):
        rm = d.rates[t]
        P.ground[t], P.excited[t], P.t1[t], P.bl[t] = rm.ground, rm.excited, rm.t1, rm.bl
        P.tau_all[t] = d.tau_all[t]
        for c, k in enumerate(ks):
            if k > 0.0:
                tauD = d.tau_all[t]
                P.tau[t][c] = tauD / (1.0 + k * tauD)
                # ground truth E (pipeline.py:414); tau_DA above is pipeline.py:415
                P.fret_E[t][c] = k * tauD / (1.0 + k * tauD)
            else:
                P.tau[t][c] = d.tau_all[t]
                P.fret_E[t][c] = 0.0
            for pss in range(2):
                if k > 0.0:
                    kb = d.k_fret_bound[t]
                    frac = min(k / kb, 1.0) if kb > 0.0 else 0.0
                    md = d.mean_ph[t, pss] * (1.0 - frac) + d.mean_ph_fret[t, pss] * frac
                    mf = d.mean_fret[t, pss] * (1.0 - frac) + d.mean_fret_fret[t, pss] * frac
                    t00 = d.T_step[t, pss, 0] * (1.0 - frac) + d.T_step_fret[t, pss, 0] * frac
                    t01 = d.T_step[t, pss, 1] * (1.0 - frac) + d.T_step_fret[t, pss, 1] * frac
                else:
                    md, mf = d.mean_ph[t, pss], d.mean_fret[t, pss]
                    t00, t01 = d.T_step[t, pss, 0], d.T_step[t, pss, 1]
                md, mf, t00, t01 = float(md), float(mf), float(t00), float(t01)
                P.mean_d[t][pss][c], P.mean_f[t][pss][c] = md, mf
                P.exp_neg_d[t][pss][c] = math.exp(-md)
                P.exp_neg_f[t][pss][c] = math.exp(-mf)
                P.T00[t][pss][c], P.T0001[t][pss][c] = t00, t00 + t01
    for c, k in enumerate(ks):
        P.has_fret_cls[c] = int(k > 0.0)
    # donors of a FRET pair with a usable lifetime get ground-truth E / tau_DA (pipeline.py:385-398)
    for fp in config.fret_pairs:
        fi = next((i for i, f in enumerate(config.fluorophores) if f.name == fp.donor_type), None)
        if fi is not None and fi < d.n_fluoro and 0.0 < d.tau_all[fi] < math.inf:
            P.gt_donor[fi] = 1
    P.donor_channel, P.acceptor_channel = d.donor_channel, d.acceptor_channel
    P.max_photons, P.est_photons = d.max_photons, d.est_photons
    P.photon_offset, P.emitter_offset, P.n_emitters = photon_offset, emitter_offset, n_emitters
    return P, d


# ----------------------------------------------------------------------------
# Microscope constants (microscope.py:97-151, 259-285, 660-714, 830-837)
# ----------------------------------------------------------------------------
@dataclass
class ScopeDerived:
    sigma_um: Dict[int, float] = field(default_factory=dict)
    fwhm_um: Dict[int, float] = field(default_factory=dict)
    pixel_size_um: float = 0.0
    offset_x: float = 0.0
    offset_y: float = 0.0
    psf_range_px: int = 0
    n_channels: int = 2
    bin_width: float = 0.0
    sigma_irf: float = 0.0
    frame_shape: Tuple[int, int, int, int] = (0, 0, 0, 0)


def build_scope_params(config: SimulationConfig, flim_offset: int = 0) -> Tuple[EdmScopeParams, ScopeDerived]:
    d = ScopeDerived()
    NA = config.objective.NA
    for ch, fluo in enumerate(config.fluorophores):
        lam_em = config.psf.emission_wavelength
        for st in fluo.states:
            if st.is_fluorescent and st.emission_wavelength > 0:
                lam_em = st.emission_wavelength
                break
        s_ill = 0.21 * config.laser.wavelength / NA
        s_det = 0.21 * lam_em / NA
        s_conf = 1.0 / math.sqrt(1.0 / (s_ill ** 2) + 1.0 / (s_det ** 2))
        su = s_conf / 1000.0
        d.sigma_um[ch] = su
        d.fwhm_um[ch] = su * 2.0 * math.sqrt(2.0 * math.log(2.0))
    d.pixel_size_um = config.scan.pixel_size / 1000.0
    Lx, Ly = config.membrane.size
    d.offset_x = (Lx - config.scan.pixels_x * d.pixel_size_um) / 2.0
    d.offset_y = (Ly - config.scan.pixels_y * d.pixel_size_um) / 2.0
    max_sigma = max(d.sigma_um.values()) if d.sigma_um else 0.1
    d.psf_range_px = int(math.ceil(4.0 * max_sigma / d.pixel_size_um))
    d.n_channels = max(2, len(config.fluorophores))
    d.bin_width = config.tcspc.bin_width
    f2s = 1.0 / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    d.sigma_irf = math.sqrt((config.laser.pulse_width * f2s) ** 2 + config.detector.timing_jitter ** 2)
    d.frame_shape = (d.n_channels, config.scan.pixels_x, config.scan.pixels_y, config.tcspc.n_bins)

    P = EdmScopeParams()
    P.nx, P.ny, P.n_bins, P.n_channels = config.scan.pixels_x, config.scan.pixels_y, config.tcspc.n_bins, d.n_channels
    P.psf_range_px = d.psf_range_px
    n_sig = max((max(d.sigma_um.keys()) + 1) if d.sigma_um else 1, 2)
    if n_sig > MAX_FLUO:
        raise ConfigError(f"at most {MAX_FLUO} fluorophores")
    P.n_sigma = n_sig
    sig = [0.0] * MAX_FLUO
    for ch, s in d.sigma_um.items():
        sig[ch] = s
    for ch in range(MAX_FLUO):
        s = sig[ch] if ch < n_sig else 0.0
        P.sigma_ch[ch] = s
        eff = s if s > 0.0 else sig[0]
        P.inv_2sig2_ch[ch] = 0.5 / (eff * eff) if eff > 0 else 0.0
    P.pixel_size, P.offset_x, P.offset_y = d.pixel_size_um, d.offset_x, d.offset_y
    P.bin_width, P.sigma_irf = d.bin_width, d.sigma_irf
    P.qe = config.detector.detection_efficiency
    lam = config.detector.dark_count_rate * config.scan.dwell_time * max(1, 1)
    P.dark_lambda = lam
    P.dark_exp_neg = math.exp(-lam)
    P.ap_prob = config.detector.afterpulsing_prob
    P.flim_offset = flim_offset
    return P, d
