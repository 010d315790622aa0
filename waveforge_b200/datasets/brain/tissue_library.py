"""Frequency-dependent tissue dielectric properties: the four-pole Cole-Cole
model of Gabriel, Lau & Gabriel (Phys. Med. Biol. 41:2251, 1996).

Drop-in for src/datasets/brain/tissue_library.py.  The parameter table is
the published one (the same numbers the reference tabulates at
tissue_library.py:182-268); the permittivity is evaluated with the same
complex-arithmetic steps (tissue_library.py:66-134), so (eps_r, sigma) are
bit-identical to the reference's and the painted coefficients match.

    eps*(w) = eps_inf + sum_n de_n / (1 + (j w tau_n)^(1 - alpha_n))
              + sigma_s / (j w eps0)
    eps_r = max(Re eps*, 1),  sigma = max(-Im eps* . w . eps0, 0)
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

EPS0 = 8.8541878128e-12
MU0 = 1.2566370614e-6


@dataclass(frozen=True)
class ColeColeParams:
    """Four relaxation poles (delta_eps, tau [s], alpha) plus eps_inf and the
    static conductivity sigma_s [S/m] (tissue_library.py:38-63)."""

    name: str
    eps_inf: float
    sigma_s: float
    delta_eps_1: float
    tau_1: float
    alpha_1: float
    delta_eps_2: float
    tau_2: float
    alpha_2: float
    delta_eps_3: float
    tau_3: float
    alpha_3: float
    delta_eps_4: float
    tau_4: float
    alpha_4: float

    def poles(self) -> tuple:
        return ((self.delta_eps_1, self.tau_1, self.alpha_1),
                (self.delta_eps_2, self.tau_2, self.alpha_2),
                (self.delta_eps_3, self.tau_3, self.alpha_3),
                (self.delta_eps_4, self.tau_4, self.alpha_4))


def _tissue(name, eps_inf, sigma_s, *poles) -> ColeColeParams:
    """Build a parameter set from (delta_eps, tau, alpha) triples."""
    flat = [v for p in poles for v in p]
    return ColeColeParams(name, eps_inf, sigma_s, *flat)


# Gabriel 1996 table II (tissues used by the brain phantom and its neighbours)
TISSUES: dict[str, ColeColeParams] = {
    "scalp": _tissue("scalp (wet skin)", 4.0, 0.0002,
                     (32.0, 7.23e-12, 0.0), (1100.0, 32.48e-9, 0.2),
                     (0.0, 159.15e-6, 0.2), (0.0, 15.92e-3, 0.2)),
    "skull_cortical": _tissue("skull (cortical bone)", 2.5, 0.02,
                              (10.0, 13.26e-12, 0.2), (180.0, 79.58e-9, 0.2),
                              (5e4, 159.15e-6, 0.2), (1e5, 15.92e-3, 0.0)),
    "csf": _tissue("cerebrospinal fluid", 4.0, 2.0,
                   (65.0, 7.96e-12, 0.1), (40.0, 1.59e-9, 0.0),
                   (0.0, 159.15e-6, 0.2), (0.0, 15.92e-3, 0.0)),
    "gray_matter": _tissue("brain gray matter", 4.0, 0.02,
                           (45.0, 7.96e-12, 0.1), (400.0, 15.92e-9, 0.15),
                           (2e5, 106.1e-6, 0.22), (4.5e7, 5.31e-3, 0.0)),
    "white_matter": _tissue("brain white matter", 4.0, 0.02,
                            (32.0, 7.96e-12, 0.1), (100.0, 7.96e-9, 0.1),
                            (4e4, 53.05e-6, 0.3), (3.5e7, 7.96e-3, 0.02)),
    "blood": _tissue("blood (fresh, oxygenated)", 4.0, 0.7,
                     (56.0, 8.38e-12, 0.1), (5200.0, 132.63e-9, 0.1),
                     (0.0, 159.15e-6, 0.2), (0.0, 15.92e-3, 0.0)),
    "dura": _tissue("dura mater", 4.0, 0.5,
                    (40.0, 7.96e-12, 0.1), (120.0, 15.92e-9, 0.15),
                    (3e4, 159.15e-6, 0.2), (3e7, 15.92e-3, 0.0)),
    "muscle": _tissue("muscle", 4.0, 0.2,
                      (50.0, 7.23e-12, 0.1), (7000.0, 353.68e-9, 0.1),
                      (1.2e6, 318.31e-6, 0.1), (2.5e7, 2.27e-3, 0.0)),
    "fat": _tissue("fat (adipose)", 2.5, 0.01,
                   (3.0, 23.0e-12, 0.2), (15.0, 159.15e-9, 0.1),
                   (3.3e4, 159.15e-6, 0.05), (1e7, 7.96e-3, 0.01)),
}

# Blood by age of the haemorrhage (tissue_library.py:246-268): fresh blood,
# then lower water content and conductivity as the clot retracts.
BLOOD_AGING: dict[str, ColeColeParams] = {
    "acute": TISSUES["blood"],
    "subacute": _tissue("blood (subacute, 6h-3d)", 4.0, 0.5,
                        (46.0, 8.38e-12, 0.1), (4000.0, 132.63e-9, 0.1),
                        (0.0, 159.15e-6, 0.2), (0.0, 15.92e-3, 0.0)),
    "chronic": _tissue("blood (chronic clot, >3d)", 4.0, 0.35,
                       (38.0, 8.38e-12, 0.1), (3000.0, 132.63e-9, 0.15),
                       (0.0, 159.15e-6, 0.2), (0.0, 15.92e-3, 0.0)),
}


def cole_cole_eps(tissue: ColeColeParams, freq_hz: float) -> complex:
    """Complex relative permittivity eps' - j eps'' at ``freq_hz``
    (tissue_library.py:66-106): empty poles are skipped, the ionic term is
    added only for sigma_s > 0 and a non-zero frequency."""
    w = 2.0 * math.pi * freq_hz
    eps = complex(tissue.eps_inf, 0.0)
    for de, tau, alpha in tissue.poles():
        if de == 0.0:
            continue
        eps += de / (1.0 + (1j * w * tau) ** (1.0 - alpha))
    if tissue.sigma_s > 0 and w > 0:
        eps += tissue.sigma_s / (1j * w * EPS0)
    return eps


def cole_cole_to_fdtd(tissue: ColeColeParams, freq_hz: float) -> tuple[float, float]:
    """(eps_r, effective sigma [S/m]) for a narrow-band solve centred at
    ``freq_hz`` (tissue_library.py:109-134): eps_r at least 1, sigma at
    least 0."""
    eps = cole_cole_eps(tissue, freq_hz)
    w = 2.0 * math.pi * freq_hz
    return max(eps.real, 1.0), max(-eps.imag * w * EPS0, 0.0)


def cole_cole_spectrum(tissue: ColeColeParams, freq_min: float = 1e8, freq_max: float = 10e9,
                       n_points: int = 200) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(frequencies, eps_r, sigma) on a log-spaced band (tissue_library.py:137-158)."""
    f = np.logspace(np.log10(freq_min), np.log10(freq_max), n_points)
    out = np.array([cole_cole_to_fdtd(tissue, x) for x in f]).reshape(n_points, 2)
    return f, out[:, 0].copy(), out[:, 1].copy()


def tissue_at_freq(name: str, freq_hz: float) -> tuple[float, float]:
    """(eps_r, sigma) of a tissue or blood-age stage by name
    (tissue_library.py:271-306); KeyError for an unknown name."""
    table = TISSUES.get(name) or BLOOD_AGING.get(name)
    if table is None:
        raise KeyError(f"Unknown tissue '{name}'. Available: "
                       f"{list(TISSUES) + list(BLOOD_AGING)}")
    return cole_cole_to_fdtd(table, freq_hz)


def all_tissues_at_freq(freq_hz: float) -> dict[str, tuple[float, float]]:
    """Every tissue, plus the blood stages as ``blood_<age>``
    (tissue_library.py:309-323)."""
    out = {name: cole_cole_to_fdtd(p, freq_hz) for name, p in TISSUES.items()}
    out.update({f"blood_{name}": cole_cole_to_fdtd(p, freq_hz) for name, p in BLOOD_AGING.items()})
    return out
