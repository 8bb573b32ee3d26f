"""Mechanism descriptions for the batched integrators.

accelerInt compiles its right-hand side into the library: the reference's
van der Pol example (``examples/van_der_pol/dydt.c:88-95``,
``examples/van_der_pol/jacob.c:129-141``) and pyJac-generated chemistry in
``mechanism/`` (absent from the reference repository).  This module provides
the two mechanism families the library evaluates on the device:

* ``VanDerPol`` -- the reference example, ``N = 2``, the parameter ``var`` is mu.
* ``MassAction`` -- a seeded synthetic constant-pressure ideal-gas mechanism
  with ``K`` species and ``R`` reversible reactions, state ``y = [T, Y_1..Y_K]``
  (``N = K + 1``), parameter ``var`` = pressure in Pa.

Mass-action model (SI for thermodynamics, CGS concentrations for kinetics):

* ``S = sum_k Y_k / W_k`` [mol/kg], ``c0 = 1e-6 * P / (R_u T)`` [mol/cm^3]
* ``C_k = c0 * (Y_k / W_k) / S`` [mol/cm^3]
* ``kf_r = exp(ln A_r + beta_r ln T - Ta_r / T)``, ``Ta = Ea / R_cal``
* ``g_k / (R_u T) = h_k / (R_u T) - s_k / R_u`` with
  ``h_k = hf_k + cp_k (T - 298.15)``, ``s_k = s0_k + cp_k ln(T / 298.15)``
* ``kr_r = kf_r * exp(dG_r / (R_u T)) * (1e-6 P_atm / (R_u T))^(-dnu_r)``
* ``q_r = kf_r prod_reac C - kr_r prod_prod C``, ``wdot_k = sum_r nu_kr q_r``
* ``dY_k/dt = W_k S wdot_k / c0``; ``dT/dt = -(S / (c0 cp_m)) sum_k h_k wdot_k``,
  ``cp_m = sum_k Y_k cp_k / W_k``.

The generator draws reactions with 1-2 reactants and 1-2 products (distinct
species), ``A`` log-uniform in [1e6, 1e14] ((cm^3/mol)^(n-1)/s), ``beta``
uniform in [-1, 1], ``Ea`` uniform in [0, 40000] cal/mol.  To keep the model
physical (mass and enthalpy conserved, so ``sum Y = 1`` and ``T`` stays
bounded), every species is a cluster of ``n_k in {1..4}`` units of one
element and reactions are drawn uniformly among the unit-conserving ones.
Species data: ``W = 16 n_k`` g/mol, ``cp = 15 + 10 n_k + U[-5, 5]`` J/mol/K,
``hf = -100 (n_k - 1) + U[-20, 20]`` kJ/mol (a 100 kJ/mol bond per
association), ``s0 = 100 + 40 n_k + U[-10, 10]`` J/mol/K (associations
lose about 100 J/mol/K), so associations are favoured below
about 1000 K and dissociations above it.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

R_UNIVERSAL = 8.31446261815324      # J/mol/K
R_CAL = 1.987204258640832           # cal/mol/K
P_ATM = 101325.0                    # Pa
T_REF = 298.15                      # K

MECH_VAN_DER_POL = 0
MECH_MASS_ACTION = 1


@dataclass
class VanDerPol:
    """The reference's van der Pol example: y0' = y1, y1' = mu (1 - y0^2) y1 - y0."""
    kind: int = MECH_VAN_DER_POL
    n_state: int = 2

    @property
    def name(self) -> str:
        return "van_der_pol"


@dataclass
class MassAction:
    """Table form of a synthetic mass-action mechanism (see the module docstring)."""
    mw: np.ndarray          # [K] kg/mol
    cp: np.ndarray          # [K] J/mol/K
    h_form: np.ndarray      # [K] J/mol at 298.15 K
    s_ref: np.ndarray       # [K] J/mol/K at 298.15 K
    reac: np.ndarray        # [R, 2] int32 species index or -1
    prod: np.ndarray        # [R, 2] int32 species index or -1
    log_a: np.ndarray       # [R] ln A
    beta: np.ndarray        # [R]
    ta: np.ndarray          # [R] activation temperature Ea / R_cal [K]
    seed: int = -1
    kind: int = MECH_MASS_ACTION
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_species(self) -> int:
        return int(self.mw.shape[0])

    @property
    def n_reactions(self) -> int:
        return int(self.log_a.shape[0])

    @property
    def n_state(self) -> int:
        return self.n_species + 1

    @property
    def name(self) -> str:
        return f"mass_action_k{self.n_species}_r{self.n_reactions}_s{self.seed}"

    def as_struct(self) -> "MassActionDesc":
        """Plain-pointer view matching ``accelerInt_mass_action`` in include/accelerint_b200.h."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (self.mw, self.cp, self.h_form, self.s_ref, self.log_a, self.beta, self.ta)]
        ints = [np.ascontiguousarray(a, dtype=np.int32).reshape(-1) for a in (self.reac, self.prod)]
        self._keep[:] = arrs + ints
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        d = MassActionDesc()
        d.n_species = self.n_species
        d.n_reactions = self.n_reactions
        d.mw, d.cp, d.h_form, d.s_ref, d.log_a, d.beta, d.ta = [a.ctypes.data_as(dp) for a in arrs]
        d.reac, d.prod = [a.ctypes.data_as(ip) for a in ints]
        return d


class MassActionDesc(ctypes.Structure):
    """ctypes mirror of ``accelerInt_mass_action`` (include/accelerint_b200.h)."""
    _fields_ = [
        ("n_species", ctypes.c_int),
        ("n_reactions", ctypes.c_int),
        ("mw", ctypes.POINTER(ctypes.c_double)),
        ("cp", ctypes.POINTER(ctypes.c_double)),
        ("h_form", ctypes.POINTER(ctypes.c_double)),
        ("s_ref", ctypes.POINTER(ctypes.c_double)),
        ("reac", ctypes.POINTER(ctypes.c_int)),
        ("prod", ctypes.POINTER(ctypes.c_int)),
        ("log_a", ctypes.POINTER(ctypes.c_double)),
        ("beta", ctypes.POINTER(ctypes.c_double)),
        ("ta", ctypes.POINTER(ctypes.c_double)),
    ]


def synthetic_mechanism(n_species: int, n_reactions: int, seed: int) -> MassAction:
    """Draw the seeded synthetic mechanism (13/27 for the 14-state workload, 53/325 for 54)."""
    rng = np.random.default_rng(seed)
    K, R = int(n_species), int(n_reactions)
    units = np.concatenate([np.arange(1, 5), rng.integers(1, 5, K - 4)])  # every size present
    rng.shuffle(units)
    mw = 16.0e-3 * units
    cp = 15.0 + 10.0 * units + rng.uniform(-5.0, 5.0, K)
    h_form = -100e3 * (units - 1) + rng.uniform(-20e3, 20e3, K)
    s_ref = 100.0 + 40.0 * units + rng.uniform(-10.0, 10.0, K)
    reac = -np.ones((R, 2), dtype=np.int32)
    prod = -np.ones((R, 2), dtype=np.int32)
    r = 0
    while r < R:
        nr = int(rng.integers(1, 3))
        npr = int(rng.integers(1, 3))
        re = rng.choice(K, nr, replace=False)
        total = int(units[re].sum())
        rest = np.setdiff1d(np.arange(K), re)
        if npr == 1:
            cand = [(int(a),) for a in rest if units[a] == total]
        else:
            cand = [(int(a), int(b)) for i, a in enumerate(rest) for b in rest[i + 1:]
                    if units[a] + units[b] == total]
        if not cand:
            continue
        pr = cand[int(rng.integers(0, len(cand)))]
        reac[r, :nr] = re
        prod[r, :npr] = pr
        r += 1
    log_a = np.log(10.0) * rng.uniform(6.0, 14.0, R)
    beta = rng.uniform(-1.0, 1.0, R)
    ea = rng.uniform(0.0, 40000.0, R)
    return MassAction(mw=mw, cp=cp, h_form=h_form, s_ref=s_ref, reac=reac, prod=prod,
                      log_a=log_a, beta=beta, ta=ea / R_CAL, seed=int(seed))


# Seeds of the published workloads: one mechanism per size, ICs drawn separately.
MECH13_SEED = 1301
MECH53_SEED = 5301


def mechanism_13() -> MassAction:
    """13 species, 27 reversible reactions (state length 14)."""
    return synthetic_mechanism(13, 27, MECH13_SEED)


def mechanism_53() -> MassAction:
    """53 species, 325 reversible reactions (state length 54)."""
    return synthetic_mechanism(53, 325, MECH53_SEED)


# ---------------------------------------------------------------- initial conditions

def vdp_initial_conditions(num: int, seed: int = 0):
    """y1 ~ U[-2, 2], y2 ~ U[-1, 1], mu = 1000.  Returns (y[N, num] column-major, var[num])."""
    rng = np.random.default_rng(seed)
    y = np.empty((2, num))
    y[0] = rng.uniform(-2.0, 2.0, num)
    y[1] = rng.uniform(-1.0, 1.0, num)
    var = np.full(num, 1000.0)
    return y, var


def _dirichlet_mass_fractions(rng, mech: MassAction, num: int) -> np.ndarray:
    x = rng.dirichlet(np.full(mech.n_species, 0.5), size=num)          # [num, K]
    yk = x * mech.mw[None, :]
    yk /= yk.sum(axis=1, keepdims=True)
    return yk.T                                                         # [K, num]


def mass_action_initial_conditions(mech: MassAction, num: int, seed: int,
                                   t_lo: float = 1000.0, t_hi: float = 1600.0,
                                   pressure: float = P_ATM):
    """T ~ U[t_lo, t_hi], P fixed, mole fractions ~ Dirichlet(0.5) converted to mass fractions."""
    rng = np.random.default_rng(seed)
    y = np.empty((mech.n_state, num))
    y[0] = rng.uniform(t_lo, t_hi, num)
    y[1:] = _dirichlet_mass_fractions(rng, mech, num)
    return y, np.full(num, pressure)


def equilibrium_mole_fractions(mech: MassAction, T: np.ndarray, pressure: float = P_ATM) -> np.ndarray:
    """Chemical equilibrium at fixed T, P of the one-element cluster mechanism.

    With unit counts n_k, equilibrium means mu_k = n_k * lam for every species, i.e.
    x_k = (P_atm / P) exp((n_k lam - g_k(T)) / (R T)); lam solves sum_k x_k = 1
    (monotone in lam, found by bisection).  Returns x[K, num]."""
    T = np.atleast_1d(np.asarray(T, dtype=np.float64))
    units = np.round(mech.mw / 16.0e-3)
    h = mech.h_form[:, None] + mech.cp[:, None] * (T[None, :] - T_REF)
    s = mech.s_ref[:, None] + mech.cp[:, None] * np.log(T[None, :] / T_REF)
    g_rt = h / (R_UNIVERSAL * T[None, :]) - s / R_UNIVERSAL             # [K, num]
    lnp = np.log(P_ATM / pressure)

    def logsum(lam):
        a = units[:, None] * lam[None, :] - g_rt + lnp
        m = a.max(axis=0)
        return m + np.log(np.exp(a - m).sum(axis=0))

    lo = np.full(T.shape, -1e3)
    hi = np.full(T.shape, 1e3)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        pos = logsum(mid) > 0.0
        hi = np.where(pos, mid, hi)
        lo = np.where(pos, lo, mid)
    lam = 0.5 * (lo + hi)
    x = np.exp(units[:, None] * lam[None, :] - g_rt + lnp)
    return x / x.sum(axis=0, keepdims=True)


def mixed_stiffness_initial_conditions(mech: MassAction, num: int, seed: int,
                                       pressure: float = P_ATM, perturbation: float = 0.05):
    """Half near-equilibrium and half ignition systems, interleaved (even index: near
    equilibrium, odd index: ignition) so queue order is not sorted by stiffness.

    near equilibrium: T ~ U[800, 1200] K, equilibrium mole fractions at that T with a
                      log-normal perturbation of relative size ``perturbation``;
    ignition:         T ~ U[1400, 2400] K, mole fractions ~ Dirichlet(0.5)."""
    rng = np.random.default_rng(seed)
    y = np.empty((mech.n_state, num))
    lo = rng.uniform(800.0, 1200.0, num)
    hi = rng.uniform(1400.0, 2400.0, num)
    even = np.arange(num) % 2 == 0
    y[0] = np.where(even, lo, hi)
    y[1:] = _dirichlet_mass_fractions(rng, mech, num)
    ne = np.flatnonzero(even)
    if ne.size:
        x = equilibrium_mole_fractions(mech, y[0, ne], pressure)
        x = x * np.exp(perturbation * rng.standard_normal(x.shape))
        yk = x * mech.mw[:, None]
        y[1:, ne] = yk / yk.sum(axis=0, keepdims=True)
    return y, np.full(num, pressure)
