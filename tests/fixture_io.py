"""Writes a parity case as a CSV fixture directory in libuw12's test_data layout
(tests/test_data.hpp:100-140 of the reference): W2/W3/W3_ri, V2/V3/V3_ri,
WV2/WV3, S, orbitals and occ (or their _alpha/_beta pairs), n_active_<suffix>
and, when given, the expected energy_<suffix> and fock (fock_alpha/_beta)."""
from pathlib import Path

import numpy as np


def _save(path: Path, a):
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a[:, None]
    np.savetxt(path, a, delimiter=",", fmt="%.16e")


def write_fixture(d, directory: Path, suffix: str, energy=None, fock=None):
    directory.mkdir(parents=True, exist_ok=True)
    for name in ("W3", "W2", "W3_ri", "V3", "V2", "V3_ri", "WV3", "WV2", "S"):
        _save(directory / f"{name}.csv", getattr(d, name))
    n_spin = len(d.orbitals)
    names = [""] if n_spin == 1 else ["_alpha", "_beta"]
    for s, nm in enumerate(names):
        _save(directory / f"orbitals{nm}.csv", d.orbitals[s])
        _save(directory / f"occ{nm}.csv", d.occ[s])
        if fock is not None:
            _save(directory / f"fock{nm}.csv", fock[s])
    np.savetxt(directory / f"n_active_{suffix}.csv", np.asarray([list(d.case.n_active)]),
               delimiter=",", fmt="%d")
    if energy is not None:
        _save(directory / f"energy_{suffix}.csv", [energy])
