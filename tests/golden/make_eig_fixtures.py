#!/usr/bin/env python
"""Generate the FP64 oracle eigenpair fixtures used by tests/test_gpu_oracle_eigs.py.

For each case below, the oracle alone (oracle/momed_oracle.c: the reference's basis
enumeration, scatter-list builders, CPU map and FP64 Lanczos restated) enumerates the mesh's
sectors, builds H(u) = H0 + u V of the synthetic recipe, and solves one sector for nev + 2
eigenpairs at tol 1e-12 (the two extra values give the gap below the unwanted spectrum).
Stored per case: the eigenvalues, each wanted eigenvector's residual ||H psi - E psi|| (the
oracle's own FP64 map), and an eigenvector sketch: the inner products r_j^H psi with 8 unit-norm
complex Gaussian probes r_j from numpy's frozen legacy generator RandomState(SKETCH_SEED)
(real parts of all 8 probes first, then imaginary parts), so a test can estimate the overlap of
a GPU eigenvector with the oracle's without storing vectors.

    python tests/golden/make_eig_fixtures.py [case ...]     # default: every case (tens of minutes)

The cases are the benchmark configurations at their full sizes: the 3x9 U0 sweep (3 U0 values
on one sector, one on another), one ~1.0M-state 3x10 sector (nev 6, krylovdim 64), and, for the
two-component configuration, a 4x5 (3+3) sector: the 4x6 (4+4) sector of ~4.7M states takes the
oracle's gather map (O(N x terms) per map) many hours on a host, so the smaller two-component
sector of the same recipe stands in for it.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

SKETCH_SEED = 1234
N_PROBES = 8
U_GRID = 0.5 + 1.5 * np.arange(32) / 31          # the sweep's 32 U0 values

CASES = {
    "c3_3x9_s3_u0": dict(a=3, b=9, N_each=(9,), seed=2, ncc=1, sector=3, u=float(U_GRID[0]), nev=4, kd=30),
    "c3_3x9_s3_u15": dict(a=3, b=9, N_each=(9,), seed=2, ncc=1, sector=3, u=float(U_GRID[15]), nev=4, kd=30),
    "c3_3x9_s3_u31": dict(a=3, b=9, N_each=(9,), seed=2, ncc=1, sector=3, u=float(U_GRID[31]), nev=4, kd=30),
    "c3_3x9_s16_u7": dict(a=3, b=9, N_each=(9,), seed=2, ncc=1, sector=16, u=float(U_GRID[7]), nev=4, kd=30),
    "c2_3x10_s3": dict(a=3, b=10, N_each=(10,), seed=1, ncc=1, sector=3, u=1.0, nev=6, kd=64),
    "c4_4x5_3p3_s5": dict(a=4, b=5, N_each=(3, 3), seed=3, ncc=2, sector=5, u=1.0, nev=8, kd=30),
}


def sketch_probes(N: int) -> np.ndarray:
    rs = np.random.RandomState(SKETCH_SEED)
    re = rs.standard_normal((N_PROBES, N))
    im = rs.standard_normal((N_PROBES, N))
    r = re + 1j * im
    return r / np.linalg.norm(r, axis=1, keepdims=True)


def operator(a, b, seed, ncc, u):
    """Hermitian-completed term list of H0 + u V (the union of both completed lists)."""
    S = O.Synth(a, b, seed, Nc_conserve=ncc)
    one = O.hermitian_complete(O.sort_merge(S.onebody()))
    two = O.hermitian_complete(O.sort_merge(S.twobody()))
    keys = np.concatenate([one[["out", "in"]], two[["out", "in"]]])
    uk, inv = np.unique(keys, return_inverse=True)
    amp = np.zeros(len(uk), np.complex128)
    amp_b = np.zeros(len(uk), np.complex128)
    np.add.at(amp, inv[:len(one)], one["re"] + 1j * one["im"])
    np.add.at(amp_b, inv[len(one):], two["re"] + 1j * two["im"])
    amp = amp + u * amp_b
    pm = np.zeros(len(uk), np.uint64)
    pm[inv[:len(one)]] = one["pm"]
    pm[inv[len(one):]] = two["pm"]
    full = np.zeros(len(uk), O.SCAT_DTYPE)
    full["re"], full["im"], full["out"], full["in"], full["pm"] = amp.real, amp.imag, uk["out"], uk["in"], pm
    return full


def run_case(name: str, c: dict) -> dict:
    t0 = time.perf_counter()
    a, b = c["a"], c["b"]
    bases, ks = O.momentum_subspaces(O.mesh_klist(a, b), (a, b), c["N_each"], Nc_conserve=c["ncc"])
    basis = bases[c["sector"]]
    full = operator(a, b, c["seed"], c["ncc"], c["u"])
    nthreads = os.cpu_count() or 1
    nev = c["nev"]
    vals, vecs, _, info = O.eigsolve(basis, full, nev + 2, krylovdim=c["kd"], tol=1e-12, maxiter=300, seed=1,
                                     nthreads=nthreads, want_vectors=True)
    resid = []
    for i in range(nev):
        y = O.matvec(basis, full, vecs[i], nthreads=nthreads)
        resid.append(float(np.linalg.norm(y - vals[i] * vecs[i])))
    R = sketch_probes(len(basis))
    sk = R.conj() @ vecs[:nev].T                    # [probe][vector]
    out = dict(case=name, mesh=[a, b], N_each=list(c["N_each"]), seed=c["seed"], Nc_conserve=c["ncc"],
               sector=c["sector"], k=[int(v) for v in ks[c["sector"]]], N=len(basis), u=c["u"], nev=nev,
               krylovdim=c["kd"], tol=1e-12, vals=[float(v) for v in vals], resid=resid,
               sketch_seed=SKETCH_SEED, sketch_re=sk.real.T.tolist(), sketch_im=sk.imag.T.tolist(),
               oracle_matvecs=int(info["matvecs"]), oracle_converged=int(info["converged"]),
               oracle_seconds=round(time.perf_counter() - t0, 1), oracle_threads=nthreads)
    return out


def main():
    names = sys.argv[1:] or list(CASES)
    path = os.path.join(HERE, "eig_oracle.json")
    data = json.load(open(path)) if os.path.exists(path) else {}
    for n in names:
        res = run_case(n, CASES[n])
        data[n] = res
        print(f"{n}: N={res['N']} vals={res['vals'][:res['nev']]} resid<={max(res['resid']):.2e} "
              f"{res['oracle_seconds']} s", flush=True)
        with open(path, "w") as f:
            json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
