"""Regenerates the golden fixtures under tests/golden/ from the reference.

Run with the path of a reference checkout (an argument, or the
RSATB_REFERENCE environment variable; there is no default):

    python tests/golden/make_golden.py <reference checkout>

It writes:

* ``kpm_ref_density.npz`` -- densities from the reference's own numpy KPM
  reconstruction (examples/publication/spectrum_realspace/kpm_ref.py:
  ``jackson``, ``n_moments_for``, ``kpm_curves``) for a seeded spectrum,
  plus ``jackson(m)`` for a few m.  kpm_ref.py states that it mirrors
  rsatb/calc/kpm.hpp and observables.hpp exactly (moment count, edge
  inset, 2*rho amplitude).
* ``fftcheb_toys.json`` -- the 2x2 complex-Hermitian Greenwood and Bastin
  toy problems (H, Vx, Vy, Vz, S, two samples) of
  rsatb/calc/test/test_fftcheb_transport.cpp:78-155, read out of that file.
* ``ed_greenwood.npz`` -- the reference's exact-diagonalisation Kubo-
  Greenwood sum (examples/publication/transport/make_ref_curves.py:
  ``delta_matrix`` and ``window_from_cheb_grid``, the dc_spectrum reference
  of ``ref_dc_spectrum``) on a seeded 40-orbital tight-binding chain with a
  bond-current velocity: sum_nm |V_nm|^2 dJ(E_k - e_n) dJ(E_k - e_m) on the
  Chebyshev-node grid, without the driver's 2 pi / Omega unit scale.

The tests only read these files; the reference tree is not needed to run
them.
"""
from __future__ import annotations

import importlib.util
import json
import math
import os
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF: Path | None = None  # the reference checkout, set from the command line


def _load(rel: str, name: str):
    spec = importlib.util.spec_from_file_location(name, REF / rel)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_kpm_ref():
    return _load("examples/publication/spectrum_realspace/kpm_ref.py", "kpm_ref")


def ed_problem(n: int = 40, seed: int = 23):
    """Seeded dense test operator for the ED transport fixture: a periodic
    chain with nearest and next-nearest hoppings and random onsite energies
    (real symmetric H), positions x_i = i, and the bond-current velocity
    V = i [H, X] restricted to the bonds (V_ij = i (x_j - x_i) H_ij with the
    periodic minimum-image distance), which is imaginary Hermitian."""
    rng = np.random.default_rng(seed)
    H = np.zeros((n, n))
    V = np.zeros((n, n), dtype=np.complex128)
    H[np.arange(n), np.arange(n)] = rng.uniform(-0.8, 0.8, n)
    for d, t0 in ((1, -1.0), (2, 0.3)):
        t = t0 + rng.uniform(-0.2, 0.2, n)
        for i in range(n):
            j = (i + d) % n
            H[i, j] = H[j, i] = t[i]
            V[i, j] = 1j * d * t[i]
            V[j, i] = -1j * d * t[i]
    return H, V


def make_ed_fixture():
    mrc = _load("examples/publication/transport/make_ref_curves.py", "make_ref_curves")
    H, V = ed_problem()
    e, U = np.linalg.eigh(H)
    W = np.abs(U.conj().T @ V @ U) ** 2
    center, half_width, M = 0.1, 3.2, 48
    k = np.arange(M)
    E = center + half_width * np.cos(np.pi * (M - 1 - k + 0.5) / M)
    c, a = mrc.window_from_cheb_grid(E)
    dJ = mrc.delta_matrix(E, e, c, a, M)
    core = np.einsum("kn,nm,km->k", dJ, W, dJ)
    np.savez(HERE / "ed_greenwood.npz", H=H, V=V, center=center, half_width=half_width,
             n_moments=M, energy=E, window=np.array([c, a]), jackson=mrc.jackson(M),
             kg_sum=core)


def make_kpm_fixture():
    kr = load_kpm_ref()
    rng = np.random.default_rng(11)
    n_states = 48
    eps = np.sort(rng.uniform(-2.3, 2.6, n_states))
    emin, emax = -3.0, 3.2
    de = 0.35
    # The run's energy grid (observables.hpp:370-375, 438-443).
    span = emax - emin
    nt = max(1, math.ceil(span / de))
    scale, shift = span / 2.0, (emax + emin) / 2.0
    i = np.arange(nt)
    energy = np.concatenate([(i - nt) * scale / nt + shift, i * scale / nt + shift])
    n_moments = kr.n_moments_for(energy, de)
    rows = np.ones((1, n_states))
    curve = kr.kpm_curves(eps, rows, energy, n_moments, n_states)[0]
    jack = {str(m): kr.jackson(m) for m in (1, 2, 7, 64, 513)}
    np.savez(HERE / "kpm_ref_density.npz", eps=eps, energy=energy, emin=emin, emax=emax, de=de,
             n_moments=n_moments, curve=curve, **{f"jackson_{k}": v for k, v in jack.items()})


_SCALAR = re.compile(r"Scalar\(([^()]*(?:\([^()]*\)[^()]*)*),\s*([^()]*(?:\([^()]*\)[^()]*)*)\)")


def _num(expr: str) -> float:
    expr = expr.strip().replace("std::sqrt", "sqrt")
    if not re.fullmatch(r"[-+*/ .0-9e()sqrt]+", expr):
        raise ValueError(f"unexpected numeric expression {expr!r}")
    return float(eval(expr, {"__builtins__": {}}, {"sqrt": math.sqrt}))


def _parse_problem(body: str) -> dict:
    out = {}
    for kind, name, block in re.findall(
            r"fill_(matrix|vector)\(\s*\*?problem\.(\w+),\s*\{(.*?)\}\s*\);", body, re.S):
        vals = [complex(_num(a), _num(b)) for a, b in _SCALAR.findall(block)]
        if kind == "matrix":
            n = int(round(math.sqrt(len(vals))))
            out[name] = [[[v.real, v.imag] for v in vals[r * n:(r + 1) * n]] for r in range(n)]
        else:
            out[name] = [[v.real, v.imag] for v in vals]
    return out


def make_fftcheb_fixture():
    src = (REF / "rsatb/calc/test/test_fftcheb_transport.cpp").read_text()
    g0 = src.index("ToyProblem make_greenwood_problem")
    b0 = src.index("ToyProblem make_bastin_problem")
    b1 = src.index("template", b0)
    fixture = {
        "source": "rsatb/calc/test/test_fftcheb_transport.cpp:78-155",
        "greenwood": _parse_problem(src[g0:b0]),
        "bastin": _parse_problem(src[b0:b1]),
    }
    (HERE / "fftcheb_toys.json").write_text(json.dumps(fixture, indent=1))


if __name__ == "__main__":
    import sys
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RSATB_REFERENCE")
    if not arg:
        sys.exit("usage: make_golden.py <reference checkout> (or set RSATB_REFERENCE)")
    REF = Path(arg)
    make_kpm_fixture()
    make_fftcheb_fixture()
    make_ed_fixture()
    print("fixtures written to", HERE)
